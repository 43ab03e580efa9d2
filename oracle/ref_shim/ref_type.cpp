/* QUICK's gpu_type.cu (basis upload helper) compiled as host code. */
#include "qref_shim.h"
#include "gpu_type.cu"
