"""quick_b200: a B200-native (sm_100a) implementation of QUICK's direct-SCF
two-electron hot path behind QUICK's Fortran-callable ``gpu_*_`` C ABI."""
