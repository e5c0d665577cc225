#include "dsmc_oracle.h"
