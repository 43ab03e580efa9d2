// Closed-shell exchange-correlation functionals of QUICK's GPU XC path
// (src/cuda/gpu_getxc.cu:144-265): B3LYP (method 1) and BLYP (method 2).
//
// Both are evaluated as f(rho, sigma) of the total density rho and
// sigma = |grad rho|^2, with the partial derivatives carried by forward-mode
// dual numbers.  The kernel needs
//     f,  f_rho = df/drho,  f_sig4 = 4 df/dsigma,
// which are QUICK's energy density, `dfdr` and `dot` (gpu_getxc.cu:175-230):
// V_ij += w [f_rho phi_i phi_j + f_sig4 grad(rho_alpha).grad(phi_i phi_j)].
//
// Formulas (restated from the publications, not from QUICK's generated code):
//  * Slater exchange: -(3/4)(3/pi)^(1/3) rho^(4/3).
//  * Becke 88 gradient correction (Phys. Rev. A 38 (1988) 3098), per spin
//    -beta rho_s^(4/3) x_s^2 / (1 + 6 beta x_s asinh x_s), beta = 0.0042,
//    x_s = |grad rho_s| / rho_s^(4/3).
//  * LYP correlation in the Miehlich-Savin-Stoll-Preuss form
//    (Chem. Phys. Lett. 157 (1989) 200), a = 0.04918, b = 0.132,
//    c = 0.2533, d = 0.349.
//  * VWN correlation with the RPA parameters (Vosko, Wilk, Nusair,
//    Can. J. Phys. 58 (1980) 1200; A = 0.0310907, x0 = -0.409286,
//    b = 13.0720, c = 42.7198), as used in B3LYP.
//  * B3LYP (Stephens et al., J. Phys. Chem. 98 (1994) 11623):
//    0.08 Slater + 0.72 B88 (B88 containing its own Slater part, so 0.80
//    Slater in all) + 0.19 VWN-RPA + 0.81 LYP; the 0.20 exact exchange is in
//    the Fock build.  BLYP: B88 + LYP.
#pragma once
#include <math.h>

namespace qb {

struct Dual2 {
    double v, dr, ds;   // value, d/drho, d/dsigma
};

__host__ __device__ __forceinline__ Dual2 mkc(double c) { return {c, 0.0, 0.0}; }
__host__ __device__ __forceinline__ Dual2 operator+(Dual2 a, Dual2 b) { return {a.v + b.v, a.dr + b.dr, a.ds + b.ds}; }
__host__ __device__ __forceinline__ Dual2 operator-(Dual2 a, Dual2 b) { return {a.v - b.v, a.dr - b.dr, a.ds - b.ds}; }
__host__ __device__ __forceinline__ Dual2 operator-(Dual2 a) { return {-a.v, -a.dr, -a.ds}; }
__host__ __device__ __forceinline__ Dual2 operator*(Dual2 a, Dual2 b)
{
    return {a.v * b.v, a.dr * b.v + a.v * b.dr, a.ds * b.v + a.v * b.ds};
}
__host__ __device__ __forceinline__ Dual2 operator*(double c, Dual2 a) { return {c * a.v, c * a.dr, c * a.ds}; }
__host__ __device__ __forceinline__ Dual2 operator*(Dual2 a, double c) { return {c * a.v, c * a.dr, c * a.ds}; }
__host__ __device__ __forceinline__ Dual2 operator+(Dual2 a, double c) { return {a.v + c, a.dr, a.ds}; }
__host__ __device__ __forceinline__ Dual2 operator+(double c, Dual2 a) { return {a.v + c, a.dr, a.ds}; }
__host__ __device__ __forceinline__ Dual2 operator-(double c, Dual2 a) { return {c - a.v, -a.dr, -a.ds}; }
__host__ __device__ __forceinline__ Dual2 operator-(Dual2 a, double c) { return {a.v - c, a.dr, a.ds}; }
__host__ __device__ __forceinline__ Dual2 operator/(Dual2 a, Dual2 b)
{
    double q = a.v / b.v;
    double ib = 1.0 / b.v;
    return {q, (a.dr - q * b.dr) * ib, (a.ds - q * b.ds) * ib};
}
__host__ __device__ __forceinline__ Dual2 operator/(double c, Dual2 b)
{
    double q = c / b.v;
    double ib = 1.0 / b.v;
    return {q, -q * b.dr * ib, -q * b.ds * ib};
}
__host__ __device__ __forceinline__ Dual2 operator/(Dual2 a, double c) { return {a.v / c, a.dr / c, a.ds / c}; }
// chain rule: g(a) with g'(a.v) = dg
__host__ __device__ __forceinline__ Dual2 chain(Dual2 a, double g, double dg) { return {g, dg * a.dr, dg * a.ds}; }
__host__ __device__ __forceinline__ Dual2 dpow(Dual2 a, double p)
{
    double g = pow(a.v, p);
    return chain(a, g, p * g / a.v);
}
__host__ __device__ __forceinline__ Dual2 dexp(Dual2 a)
{
    double g = exp(a.v);
    return chain(a, g, g);
}
__host__ __device__ __forceinline__ Dual2 dlog(Dual2 a) { return chain(a, log(a.v), 1.0 / a.v); }
__host__ __device__ __forceinline__ Dual2 datan(Dual2 a) { return chain(a, atan(a.v), 1.0 / (1.0 + a.v * a.v)); }

// h(s) = sqrt(s) asinh(sqrt(s)), smooth in s >= 0:
// h'(s) = asinh(sqrt s) / (2 sqrt s) + 1 / (2 sqrt(1 + s)), h'(0) = 1.
__host__ __device__ __forceinline__ Dual2 dxasinhx_of_sq(Dual2 s)
{
    double q = sqrt(s.v);
    double as = asinh(q);
    double h = q * as;
    double dh = (q > 1e-8 ? as / (2.0 * q) : 0.5 - s.v / 6.0) + 0.5 / sqrt(1.0 + s.v);
    return chain(s, h, dh);
}

// -(3/4)(3/pi)^(1/3) rho^(4/3)
__host__ __device__ __forceinline__ Dual2 slater_cs(Dual2 rho)
{
    const double cx = 0.73855876638202240587;   // (3/4) (3/pi)^(1/3)
    return -cx * dpow(rho, 4.0 / 3.0);
}

// B88 gradient correction, both spins, closed shell: rho_s = rho/2,
// |grad rho_s|^2 = sigma/4, so x_s^2 = 2^(2/3) sigma / rho^(8/3) and the sum
// over spins is -2^(1/3) beta sigma rho^(-4/3) / (1 + 6 beta x_s asinh x_s).
__host__ __device__ __forceinline__ Dual2 b88_gc_cs(Dual2 rho, Dual2 sigma)
{
    const double beta = 0.0042;
    const double c23 = 1.5874010519681994748;   // 2^(2/3)
    const double c13 = 1.2599210498948731648;   // 2^(1/3)
    Dual2 r43 = dpow(rho, 4.0 / 3.0);
    Dual2 xs2 = c23 * sigma / (r43 * r43);
    Dual2 den = 1.0 + 6.0 * beta * dxasinhx_of_sq(xs2);
    return -(c13 * beta) * sigma / (r43 * den);
}

// LYP (Miehlich et al. form) at rho_a = rho_b = rho/2,
// |grad rho_a|^2 = |grad rho_b|^2 = grad rho_a . grad rho_b = sigma/4.
__host__ __device__ __forceinline__ Dual2 lyp_cs(Dual2 rho, Dual2 sigma)
{
    const double a = 0.04918, b = 0.132, c = 0.2533, d = 0.349;
    const double cf = 2.8712340001881918;            // (3/10) (3 pi^2)^(2/3)
    const double c113 = 12.699208415745595;          // 2^(11/3)
    Dual2 pa = 0.5 * rho;                            // = pb
    Dual2 g = 0.25 * sigma;                          // gaa = gbb = gab
    Dual2 rm13 = dpow(rho, -1.0 / 3.0);
    Dual2 den = 1.0 + d * rm13;
    Dual2 omega = dexp(-c * rm13) / den * dpow(rho, -11.0 / 3.0);
    Dual2 delta = c * rm13 + d * rm13 / den;
    Dual2 papb = pa * pa;
    Dual2 pa83 = dpow(pa, 8.0 / 3.0);
    Dual2 grad2 = 4.0 * g;                           // |grad rho|^2 = gaa + gbb + 2 gab
    // rho_a rho_b [ 2^(11/3) C_F (pa^(8/3) + pb^(8/3)) + (47/18 - 7 delta/18) |grad rho|^2
    //   - (5/2 - delta/18)(gaa + gbb) - (delta - 11)/9 (pa/rho gaa + pb/rho gbb) ]
    Dual2 br = c113 * cf * (2.0 * pa83) + (47.0 / 18.0 - (7.0 / 18.0) * delta) * grad2
               - (2.5 - delta / 18.0) * (2.0 * g) - (delta - 11.0) / 9.0 * g;   // pa/rho = pb/rho = 1/2
    // - 2/3 rho^2 |grad rho|^2 + (2/3 rho^2 - pa^2) gbb + (2/3 rho^2 - pb^2) gaa
    Dual2 rho2 = rho * rho;
    Dual2 tail = -(2.0 / 3.0) * rho2 * grad2 + 2.0 * (((2.0 / 3.0) * rho2 - papb) * g);
    return -4.0 * a * papb / (rho * den) - a * b * omega * (papb * br + tail);
}

// VWN correlation energy per particle with the RPA parameters, in
// x = sqrt(r_s), r_s = (3 / (4 pi rho))^(1/3).
__host__ __device__ __forceinline__ Dual2 vwn_rpa_eps(Dual2 rho)
{
    const double A = 0.0310907, x0 = -0.409286, bb = 13.0720, cc = 42.7198;
    const double Q = 0.044899888641287296;           // sqrt(4 cc - bb^2)
    const double X0 = x0 * x0 + bb * x0 + cc;
    const double k16 = 0.78762331789974325;          // (3 / (4 pi))^(1/6)
    Dual2 x = k16 * dpow(rho, -1.0 / 6.0);
    Dual2 X = x * x + bb * x + cc;
    Dual2 at = datan(Q / (2.0 * x + bb));
    Dual2 xm = x - x0;
    return A * (dlog(x * x / X) + (2.0 * bb / Q) * at
                - (bb * x0 / X0) * (dlog(xm * xm / X) + (2.0 * (bb + 2.0 * x0) / Q) * at));
}

// method 1: B3LYP, method 2: BLYP.  Returns f; *f_rho = df/drho,
// *f_sig4 = 4 df/dsigma.
__host__ __device__ __forceinline__ double xc_eval(int method, double rho_v, double sigma_v, double* f_rho,
                                                   double* f_sig4)
{
    Dual2 rho{rho_v, 1.0, 0.0}, sigma{sigma_v, 0.0, 1.0};
    Dual2 f;
    if (method == 1)
        f = 0.8 * slater_cs(rho) + 0.72 * b88_gc_cs(rho, sigma) + 0.19 * (rho * vwn_rpa_eps(rho))
            + 0.81 * lyp_cs(rho, sigma);
    else
        f = slater_cs(rho) + b88_gc_cs(rho, sigma) + lyp_cs(rho, sigma);
    *f_rho = f.dr;
    *f_sig4 = 4.0 * f.ds;
    return f.v;
}

}  // namespace qb
