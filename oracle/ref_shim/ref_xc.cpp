/* QUICK's XC quadrature (src/cuda/gpu_getxc.cu) compiled as host code.
 * gpu_getxc.cu launches its kernel with a bare <<<...>>> expression that a
 * host compiler cannot parse, so build_ref.py first writes a copy of that
 * file into the build directory with the launch expression replaced by a
 * qref_launch() call (nothing else is changed), and this unit includes the
 * copy. */
#include "qref_shim.h"
#include "gpu.h"
#include "gpu_getxc_host.cu"
