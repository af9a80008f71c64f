// Definitions for the names declared in ref_compat.h (test oracle build only).
#include "ref_compat.h"
bool inHBM = false;
RomeOracleNoPtr _ptr;
