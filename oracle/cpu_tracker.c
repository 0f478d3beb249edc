#include "fe_oracle.h"
