/* Empty stand-in: the MAP hot path does not call the DFTI interface. */
#ifndef ROME_ORACLE_MKL_DFTI_SHIM_H
#define ROME_ORACLE_MKL_DFTI_SHIM_H
#endif
