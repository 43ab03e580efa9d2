/* QUICK's XC quadrature (src/cuda/gpu_getxc.cu) compiled as host code.
 * gpu_getxc.cu launches its kernel with a bare <<<...>>> expression that a
 * host compiler cannot parse, so build_ref.py first writes a copy of that
 * file into the build directory with the launch expression replaced by a
 * qref_launch() call (nothing else is changed), and this unit includes the
 * copy. */
#include "qref_shim.h"
#include "gpu.h"
#include "gpu_getxc_host.cu"

/* QUICK's functional routines (gpu_getxc.cu:545-1003) at a closed-shell
   point given by the total density rho and sigma = |grad rho|^2, arranged
   the way gpu_grid_xc calls them (density = rho / 2, gax = sqrt(sigma) / 2).
   f, dfdr and dot (the factor gpu_grid_xc multiplies grad rho_alpha by) are
   returned.  method 1: b3lyp_e / b3lypf; method 2: becke_e + lyp_e with
   becke + lyp. */
extern "C" void qref_functional(int method, double rho, double sigma, double* f, double* dfdr, double* dot)
{
    double pa = 0.5 * rho, ga = 0.5 * sqrt(sigma);
    if (method == 1) {
        *f = b3lyp_e(rho, sigma);
        *dot = b3lypf(rho, sigma, dfdr);
    } else {
        *f = becke_e(pa, pa, ga, 0.0, 0.0, ga, 0.0, 0.0) + lyp_e(pa, pa, ga, 0.0, 0.0, ga, 0.0, 0.0);
        double d1, gaa1, gab1, d2, gaa2, gab2;
        becke(pa, ga, 0.0, 0.0, ga, 0.0, 0.0, &d1, &gaa1, &gab1);
        lyp(pa, pa, ga, 0.0, 0.0, ga, 0.0, 0.0, &d2, &gaa2, &gab2);
        *dfdr = d1 + d2;
        *dot = 2.0 * (gaa1 + gaa2) + (gab1 + gab2);
    }
}
