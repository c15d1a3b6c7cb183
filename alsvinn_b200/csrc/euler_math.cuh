// Device-side Euler mathematics of the cell-update hot path.
//
// Every expression keeps the evaluation order of the reference so that,
// compiled with -fmad=false and IEEE division/square root, FP64 results are
// bit-identical to alsfvm's CPU path:
//   state / extra variables  alsfvm/include/alsfvm/equation/euler/Euler.hpp:172-211
//   HLL                      alsfvm/include/alsfvm/numflux/euler/HLL.hpp:51-116
//   HLL3                     alsfvm/include/alsfvm/numflux/euler/HLL3.hpp:52-149
//   Central                  alsfvm/include/alsfvm/numflux/Central.hpp:39-56
//   WENO2                    alsfvm/include/alsfvm/reconstruction/WENO2.hpp:31-91
//   MC, MM                   alsfvm/include/alsfvm/reconstruction/MC.hpp, MM.hpp, minmod.hpp
//   WENOF2                   alsfvm/include/alsfvm/reconstruction/WENOF2.hpp
//   ENO2/3/4                 alsfvm/src/reconstruction/ENOCPU.cpp:41-267,
//                            alsfvm/src/reconstruction/ENOCoefficients.cpp:27-49
// Only the velocity component along the face normal is formed: the
// reference computes all components but uses only u[direction].
#pragma once

#include <cstdint>

namespace als {

enum Recon { RECON_NONE = 0, RECON_WENO2 = 1, RECON_ENO2 = 2, RECON_ENO3 = 3, RECON_ENO4 = 4,
             RECON_MC = 5, RECON_MM = 6, RECON_WENOF2 = 7, RECON_WENO3 = 8 };
enum Flux { FLUX_HLL = 0, FLUX_HLL3 = 1, FLUX_CENTRAL = 2, FLUX_TECNO1 = 3, FLUX_TECNO4 = 4,
            FLUX_TECNO6 = 5 };

__host__ __device__ constexpr int recon_ghosts(int recon) {
    return recon == RECON_NONE ? 1
        : (recon == RECON_WENO2 || recon == RECON_ENO2 || recon == RECON_MC || recon == RECON_MM ||
           recon == RECON_WENOF2) ? 2
        : ((recon == RECON_ENO3 || recon == RECON_WENO3) ? 3 : 4);
}

// Ghost cells the flux's stencil needs: stencil size - 1 (NumericalFluxCPU.cpp:225-231);
// TecnoCombined4/6 read {-1..2} / {-2..3} (TecnoCombined4.hpp:62-66,
// TecnoCombined6.hpp:67-71), every other flux the two-point {0, 1}.
__host__ __device__ constexpr int flux_ghosts(int flux) {
    return flux == FLUX_TECNO4 ? 3 : (flux == FLUX_TECNO6 ? 5 : 1);
}

// Stencil fluxes read the cell values themselves (reconstruction "none").
__host__ __device__ constexpr bool stencil_flux(int flux) {
    return flux == FLUX_TECNO4 || flux == FLUX_TECNO6;
}

__host__ __device__ constexpr int stage_ghosts(int recon, int flux) {
    return recon_ghosts(recon) > flux_ghosts(flux) ? recon_ghosts(recon) : flux_ghosts(flux);
}

// FP32 ensemble members are compared with the FP64 path by tolerance, not
// bit for bit, so their arithmetic may be regrouped: with ALS_F32_RECIP set,
// every group of divisions by one denominator becomes one reciprocal and
// products, and the WENO2 weights take their closed form.  This halves the
// divisions of a WENO2 + HLL3 cell-stage.  FP64 code never takes these
// branches and keeps the reference's operations in the reference's order.
#ifndef ALS_F32_RECIP
#define ALS_F32_RECIP 1
#endif
template<class R>
__host__ __device__ constexpr bool fast_recip() {
    return ALS_F32_RECIP != 0 && sizeof(R) == 4;
}

// Left/right face state of one cell along direction D.
template<class R, int NSD>
struct FaceState {
    R c[NSD + 2];   // rho, m_0..m_{NSD-1}, E
    R p;            // pressure
    R ud;           // velocity along the face normal
    R ri;           // 1 / rho (set and used only when fast_recip<R>())
};

// computeExtra (Euler.hpp:204-211): ie = E - 0.5*(m.m)/rho, u = m/rho, p = (gamma-1)*ie.
template<class R, int NSD, int D>
__device__ __forceinline__ void make_state(const R* U, R gamma, FaceState<R, NSD>& s) {
#pragma unroll
    for (int k = 0; k < NSD + 2; ++k) {
        s.c[k] = U[k];
    }
    R dot = U[1] * U[1];
    if (NSD > 1) {
        dot = dot + U[2] * U[2];
    }
    if (NSD > 2) {
        dot = dot + U[3] * U[3];
    }
    if constexpr (fast_recip<R>()) {
        const R ri = R(1) / U[0];
        s.ri = ri;
        s.ud = U[1 + D] * ri;
        s.p = (gamma - R(1)) * (U[NSD + 1] - R(0.5) * dot * ri);
    } else {
        const R ie = U[NSD + 1] - R(0.5) * dot / U[0];
        s.ud = U[1 + D] / U[0];
        s.p = (gamma - R(1)) * ie;
    }
}

// gamma p / rho of a face state (the squared sound speed).
template<class R, int NSD>
__device__ __forceinline__ R sound2(const FaceState<R, NSD>& s, R gamma) {
    if constexpr (fast_recip<R>()) {
        return gamma * s.p * s.ri;
    } else {
        return gamma * s.p / s.c[0];
    }
}

// Point flux along D (Euler.hpp:172-181).
template<class R, int NSD, int D>
__device__ __forceinline__ void point_flux(const FaceState<R, NSD>& s, R* F) {
    F[0] = s.c[1 + D];
#pragma unroll
    for (int k = 0; k < NSD; ++k) {
        F[1 + k] = s.c[1 + k] * s.ud;
    }
    F[1 + D] = F[1 + D] + s.p;
    F[NSD + 1] = (s.c[NSD + 1] + s.p) * s.ud;
}

template<class R, int NSD, int D>
__device__ __forceinline__ R flux_hll(const FaceState<R, NSD>& L, const FaceState<R, NSD>& Rt,
    R gamma, R* F) {
    constexpr int NV = NSD + 2;
    const R wl = sqrt(L.c[0]);
    const R wr = sqrt(Rt.c[0]);
    const R rho = (L.c[0] + Rt.c[0]) / R(2);
    R ud, p;
    if constexpr (fast_recip<R>()) {
        const R iw = R(1) / (wl + wr);
        ud = (wl * L.ud + wr * Rt.ud) * iw;
        p = (L.p * wl + Rt.p * wr) * iw;
    } else {
        ud = (wl * L.ud + wr * Rt.ud) / (wl + wr);
        p = (L.p * wl + Rt.p * wr) / (wl + wr);
    }
    const R cs = sqrt(gamma * p / rho);
    const R sL = fmin(L.ud - sqrt(sound2(L, gamma)), ud - cs);
    const R sR = fmax(Rt.ud + sqrt(sound2(Rt, gamma)), ud + cs);
    if (sL == R(0)) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            F[k] = R(0);
        }
    } else if (sL > R(0)) {
        point_flux<R, NSD, D>(L, F);
    } else if (sR < R(0)) {
        point_flux<R, NSD, D>(Rt, F);
    } else {
        R FL[NV], FR[NV];
        point_flux<R, NSD, D>(L, FL);
        point_flux<R, NSD, D>(Rt, FR);
        const R srsl = sR * sL;
        const R den = sR - sL;
        const R iden = fast_recip<R>() ? R(1) / den : R(0);
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            const R num = sR * FL[k] - sL * FR[k] + srsl * (Rt.c[k] - L.c[k]);
            F[k] = fast_recip<R>() ? num * iden : num / den;
        }
    }
    return fmax(fabs(sL), fabs(sR));
}

// HLL3::computeHLLSpeeds (HLL3.hpp:120-160): Roe-averaged speeds with the
// shock correction.
template<class R, int NSD>
__device__ __forceinline__ void hll3_speeds(const FaceState<R, NSD>& L, const FaceState<R, NSD>& Rt,
    R gamma, R& sL, R& sR) {
    const R wl = sqrt(L.c[0]);
    const R wr = sqrt(Rt.c[0]);
    const R rho = (L.c[0] + Rt.c[0]) / R(2);
    R ud, p;
    if constexpr (fast_recip<R>()) {
        const R iw = R(1) / (wl + wr);
        ud = (wl * L.ud + wr * Rt.ud) * iw;
        p = (wl * L.p + wr * Rt.p) * iw;
    } else {
        ud = (wl * L.ud + wr * Rt.ud) / (wl + wr);
        p = (wl * L.p + wr * Rt.p) / (wl + wr);
    }
    const R cfL = sqrt(sound2(L, gamma));
    const R cfR = sqrt(sound2(Rt, gamma));
    const R correct = R(0.5) * fmax(R(0), L.ud - Rt.ud);
    const R cs = sqrt(gamma * p / rho);
    sL = fmin(L.ud + correct - cfL, ud - cs);
    sR = fmax(Rt.ud - correct + cfR, ud + cs);
}

template<class R, int NSD, int D>
__device__ __forceinline__ R flux_hll3(const FaceState<R, NSD>& L, const FaceState<R, NSD>& Rt,
    R gamma, R* F) {
    constexpr int NV = NSD + 2;
    R sL, sR;
    hll3_speeds<R, NSD>(L, Rt, gamma, sL, sR);
    if (sL == R(0)) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            F[k] = R(0);
        }
    } else if (sL > R(0)) {
        point_flux<R, NSD, D>(L, F);
    } else if (sR < R(0)) {
        point_flux<R, NSD, D>(Rt, F);
    } else {
        // Of the two point fluxes only the transverse momentum components
        // (c[1+k] * ud, k != D: Euler.hpp:172-181 adds p along D only) enter
        // before the star side is chosen; the chosen side's full point flux
        // is formed after the choice.  Each value is the same product the
        // reference forms, so the result is unchanged, and the two flux
        // vectors are never live together.
        const R udl = L.ud - sL;
        const R udr = Rt.ud - sR;
        const R aa = udr * Rt.c[0] - udl * L.c[0];
        const R iaa = fast_recip<R>() ? R(1) / aa : R(0);
        auto over_aa = [&](R x) { return fast_recip<R>() ? x * iaa : x / aa; };
        const R sm = over_aa(Rt.c[1 + D] * udr - L.c[1 + D] * udl + Rt.p - L.p);
        // us: transverse star velocities (the normal one is sm)
        R us[NSD];
#pragma unroll
        for (int k = 0; k < NSD; ++k) {
            if (k == D) {
                us[k] = sm;
            } else {
                const R fr = Rt.c[1 + k] * Rt.ud;
                const R fl = L.c[1 + k] * L.ud;
                us[k] = over_aa(fr - fl - sR * Rt.c[1 + k] + sL * L.c[1 + k]);
            }
        }
        const bool left = sm >= R(0);
        const FaceState<R, NSD>& S = left ? L : Rt;
        const R sK = left ? sL : sR;
        const R udk = left ? udl : udr;
        R FK[NV];
        point_flux<R, NSD, D>(S, FK);
        const R den = sm - sK;
        const R iden = fast_recip<R>() ? R(1) / den : R(0);
        auto over_den = [&](R x) { return fast_recip<R>() ? x * iden : x / den; };
        R mid[NV];
        mid[0] = over_den(S.c[0] * udk);
#pragma unroll
        for (int k = 0; k < NSD; ++k) {
            mid[1 + k] = us[k] * mid[0];
        }
        const R ps = S.p + S.c[0] * (S.ud - sm) * udk;
        mid[NSD + 1] = over_den(udk * S.c[NSD + 1] + S.p * S.ud - ps * sm);
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            F[k] = FK[k] + sK * (mid[k] - S.c[k]);
        }
    }
    return fmax(fabs(sL), fabs(sR));
}

template<class R, int NSD, int D>
__device__ __forceinline__ R flux_central(const FaceState<R, NSD>& L, const FaceState<R, NSD>& Rt,
    R gamma, R* F) {
    constexpr int NV = NSD + 2;
    R FL[NV], FR[NV];
    point_flux<R, NSD, D>(L, FL);
    point_flux<R, NSD, D>(Rt, FR);
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        F[k] = R(0.5) * (FL[k] + FR[k]);
    }
    return fmax(fabs(L.ud) + sqrt(sound2(L, gamma)), fabs(Rt.ud) + sqrt(sound2(Rt, gamma)));
}

// Logarithmic mean (b - a) / (log b - log a), 0 when either difference is 0
// (tecno_utils.hpp:30-38), and F over it, 0 when that mean is 0 (:42-50).
template<class R>
__device__ __forceinline__ R log_mean(R a, R b) {
    const R d = b - a;
    const R dl = log(b) - log(a);
    if (d == R(0) || dl == R(0)) {
        return R(0);
    }
    return d / dl;
}

template<class R>
__device__ __forceinline__ R over_log_mean(R a, R b, R F) {
    const R m = log_mean(a, b);
    return m == R(0) ? R(0) : F / m;
}

// Parameter vector z = (sqrt(rho/p), sqrt(rho/p) u, sqrt(rho p))
// (Euler.hpp:290-320), from the primitive variables u = m/rho and
// p = (gamma-1)(E - 0.5 m.m/rho).
template<class R, int NSD>
__device__ __forceinline__ void tecno_z(const FaceState<R, NSD>& s, R* z) {
    const R q = sqrt(s.c[0] / s.p);
#pragma unroll
    for (int k = 0; k < NSD; ++k) {
        z[1 + k] = (s.c[1 + k] / s.c[0]) * q;
    }
    z[0] = q;
    z[NSD + 1] = sqrt(s.c[0] * s.p);
}

// Entropy-conservative flux of Fjordholm, Mishra and Tadmor (SINUM 2012,
// eq. 6.11) as the reference states it (numflux/euler/Tecno1.hpp:51-180):
// the point flux when both states are equal; otherwise built from
// arithmetic means of z and logarithmic means of z_0 and z_last.  The
// reference writes the 2-D formulas for every dimension: in 3-D the
// z-momentum flux is 0 and the z-direction flux stays 0 unless the states
// are equal.  The wave speed is max |s| of the HLL3 speeds.
template<class R, int NSD, int D>
__device__ __forceinline__ R flux_tecno1(const FaceState<R, NSD>& L, const FaceState<R, NSD>& Rt,
    R gamma, R* F) {
    constexpr int NV = NSD + 2;
    bool same = true;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        same = same && (L.c[k] == Rt.c[k]);
    }
    if (same) {
        point_flux<R, NSD, D>(L, F);
    } else if (NSD == 3 && D == 2) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            F[k] = R(0);
        }
    } else {
        R zl[NV], zr[NV];
        tecno_z<R, NSD>(L, zl);
        tecno_z<R, NSD>(Rt, zr);
        auto bar = [&](int k) { return (zl[k] + zr[k]) / R(2); };
        F[0] = bar(1 + D) * log_mean(zl[NSD + 1], zr[NSD + 1]);
#pragma unroll
        for (int k = 0; k < NSD; ++k) {
            if (NSD == 3 && k == 2) {
                F[1 + k] = R(0);
            } else if (k == D) {
                F[1 + k] = bar(NSD + 1) / bar(0) + bar(1 + D) / bar(0) * F[0];
            } else {
                F[1 + k] = bar(1 + k) / bar(0) * F[0];
            }
        }
        R e = (gamma + R(1)) / (gamma - R(1)) * over_log_mean(zl[0], zr[0], F[0]);
        e = e + bar(1) * F[1];
        if (NSD > 1) {
            e = e + bar(2) * F[2];
        }
        F[NSD + 1] = R(1) / (R(2) * bar(0)) * e;
    }
    R sL, sR;
    hll3_speeds<R, NSD>(L, Rt, gamma, sL, sR);
    return fmax(fabs(sL), fabs(sR));
}

// F(U-, U+) at one face along D.  ul = right-reconstructed value of the cell
// left of the face, ur = left-reconstructed value of the cell to its right
// (numflux_util.hpp:62-92).  Returns the face wave speed.
template<class R, int NSD, int FLUX, int D>
__device__ __forceinline__ R face_flux(const R* ul, const R* ur, R gamma, R* F) {
    FaceState<R, NSD> L, Rt;
    make_state<R, NSD, D>(ul, gamma, L);
    make_state<R, NSD, D>(ur, gamma, Rt);
    if (FLUX == FLUX_HLL) {
        return flux_hll<R, NSD, D>(L, Rt, gamma, F);
    } else if (FLUX == FLUX_HLL3) {
        return flux_hll3<R, NSD, D>(L, Rt, gamma, F);
    } else if (FLUX == FLUX_TECNO1) {
        return flux_tecno1<R, NSD, D>(L, Rt, gamma, F);
    } else {
        return flux_central<R, NSD, D>(L, Rt, gamma, F);
    }
}

// ENO coefficients c[r][j] (ENOCoefficients.cpp:27-49), each the correctly
// rounded double quotient, converted to R on use.
static __constant__ double kEno2[3][2] = {{3.0 / 2.0, -1.0 / 2.0}, {1.0 / 2.0, 1.0 / 2.0},
    {-1.0 / 2.0, 3.0 / 2.0}};
static __constant__ double kEno3[4][3] = {{11.0 / 6.0, -7.0 / 6.0, 1.0 / 3.0},
    {1.0 / 3.0, 5.0 / 6.0, -1.0 / 6.0}, {-1.0 / 6.0, 5.0 / 6.0, 1.0 / 3.0},
    {1.0 / 3.0, -7.0 / 6.0, 11.0 / 6.0}};
static __constant__ double kEno4[5][4] = {{25.0 / 12.0, -23.0 / 12.0, 13.0 / 12.0, -1.0 / 4.0},
    {1.0 / 4.0, 13.0 / 12.0, -5.0 / 12.0, 1.0 / 12.0},
    {-1.0 / 12.0, 7.0 / 12.0, 7.0 / 12.0, -1.0 / 12.0},
    {1.0 / 12.0, -5.0 / 12.0, 13.0 / 12.0, 1.0 / 4.0},
    {-1.0 / 4.0, 13.0 / 12.0, -23.0 / 12.0, 25.0 / 12.0}};

template<class R, int ORDER>
__device__ __forceinline__ R eno_coef(int r, int j) {
    if (ORDER == 2) {
        return R(kEno2[r][j]);
    } else if (ORDER == 3) {
        return R(kEno3[r][j]);
    } else {
        return R(kEno4[r][j]);
    }
}

// Reconstruction of one cell along one direction.  The stencil values come
// from a fetcher: f.at(v, o) is variable v at offset o along the direction
// (o a compile-time constant after unrolling) and f.dyn(v, o) the same for
// a run-time offset.  Writes NV left and NV right values.
//
// In WENO2, 2/d equals 2*(1/d) exactly whenever 1/d is a normal number (a
// power-of-two scaling commutes with rounding), so the second division by
// each d is replaced by a doubling; d above 2^1021 (never reached by a
// physical state) takes the division.
template<class R>
__device__ __forceinline__ R twice_reciprocal(R d, R recip) {
    const R big = sizeof(R) == 8 ? R(2.2471164185778949e307) : R(2.1267647932558654e37);
    R out;
    if (d < big) {
        out = R(2) * recip;
    } else {
        out = R(2) / d;
    }
    return out;
}

// sign and minmod (alsfvm/include/alsfvm/reconstruction/sign.hpp,
// minmod.hpp): sign is 1, 0 or -1; minmod is sign(a) times the smallest
// magnitude when all signs agree, else 0.
template<class R>
__device__ __forceinline__ R sign_of(R a) {
    return a > R(0) ? R(1) : (a == R(0) ? R(0) : R(-1));
}

template<class R>
__device__ __forceinline__ R minmod2(R a, R b) {
    return sign_of(a) == sign_of(b) ? sign_of(a) * fmin(fabs(a), fabs(b)) : R(0);
}

template<class R>
__device__ __forceinline__ R minmod3(R a, R b, R c) {
    return (sign_of(a) == sign_of(b) && sign_of(b) == sign_of(c))
        ? sign_of(a) * fmin(fabs(a), fmin(fabs(b), fabs(c))) : R(0);
}

// Primitive variables of one cell (Euler.hpp:290-297): u = m/rho,
// p = (gamma-1)(E - 0.5 m.m / rho).
template<class R, int NSD, class Fetch>
__device__ __forceinline__ void primitive_at(const Fetch& f, int o, R gamma, R& rho, R* u, R& p) {
    rho = f.at(0, o);
    R dot = f.at(1, o) * f.at(1, o);
#pragma unroll
    for (int k = 1; k < NSD; ++k) {
        dot = dot + f.at(1 + k, o) * f.at(1 + k, o);
    }
#pragma unroll
    for (int k = 0; k < NSD; ++k) {
        u[k] = f.at(1 + k, o) / rho;
    }
    const R ie = f.at(NSD + 1, o) - R(0.5) * dot / rho;
    p = (gamma - R(1)) * ie;
}

// One side of WENOF2 (WENOF2.hpp:70-121): the bounded primitive slope dP,
// the limiter a = 0.5 sqrt(R / max(R, LL)), then computeConserved of
// mid -+ a dP (Euler.hpp:236-245).
template<class R, int NSD, bool RIGHT>
__device__ __forceinline__ void wenof2_side(R w0, R w1, R gamma, const R* rho, const R (*u)[NSD],
    const R* p, R* out) {
    const R BOUND = R(1.9);
    R dr = w1 * (rho[1] - rho[0]) + w0 * (rho[2] - rho[1]);
    R du[NSD];
#pragma unroll
    for (int k = 0; k < NSD; ++k) {
        du[k] = w1 * (u[1][k] - u[0][k]) + w0 * (u[2][k] - u[1][k]);
    }
    R dp = w1 * (p[1] - p[0]) + w0 * (p[2] - p[1]);
    dr = fmax(-BOUND * rho[1], fmin(BOUND * rho[1], dr));
    dp = fmax(-BOUND * p[1], fmin(BOUND * p[1], dp));
    R dudu = du[0] * du[0];
    R umdu = u[1][0] * du[0];
#pragma unroll
    for (int k = 1; k < NSD; ++k) {
        dudu = dudu + du[k] * du[k];
        umdu = umdu + u[1][k] * du[k];
    }
    const R LL = R(0.125) * rho[1] * dudu - R(0.5) * fmin(R(0), dr * umdu) +
        R(0.5) * dr * dr * dudu / rho[1];
    const R Rr = p[1] / (gamma - R(1));
    const R a = R(0.5) * sqrt(Rr / fmax(Rr, LL));
    R pr, pu[NSD], pp;
    if (RIGHT) {
        pr = rho[1] + a * dr;
        pp = p[1] + a * dp;
    } else {
        pr = rho[1] - a * dr;
        pp = p[1] - a * dp;
    }
    R dot = R(0);
#pragma unroll
    for (int k = 0; k < NSD; ++k) {
        pu[k] = RIGHT ? u[1][k] + a * du[k] : u[1][k] - a * du[k];
        dot = k == 0 ? pu[0] * pu[0] : dot + pu[k] * pu[k];
    }
    out[0] = pr;
#pragma unroll
    for (int k = 0; k < NSD; ++k) {
        out[1 + k] = pu[k] * pr;
    }
    out[NSD + 1] = pp / (gamma - R(1)) + R(0.5) * pr * dot;
}

template<class R, int NV, int RECON, class Fetch>
__device__ __forceinline__ void reconstruct_f(const Fetch& f, R* left, R* right, R gamma) {
    if (RECON == RECON_NONE) {
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            left[v] = f.at(v, 0);
            right[v] = left[v];
        }
    } else if (RECON == RECON_WENO2) {
        const R eps = R(1e-8);
        const R i0 = f.at(0, 0);
        const R dp = f.at(0, 1) - i0;
        const R dm = i0 - f.at(0, -1);
        const R b0 = dp * dp;
        const R b1 = dm * dm;
        const R d0 = R(3) * (eps + b0) * (eps + b0);
        const R d1 = R(3) * (eps + b1) * (eps + b1);
        R w0Left, w1Left, w0Right, w1Right;
        if constexpr (fast_recip<R>()) {
            // a0L = 1/d0, a1L = 2/d1, a0R = 2/d0, a1R = 1/d1 give w0L = d1/(d1 + 2 d0),
            // w1L = 2 d0/(d1 + 2 d0), w0R = 2 d1/(2 d1 + d0), w1R = d0/(2 d1 + d0)
            // (d stays finite in FP32 while neighbouring densities differ by < 1e9)
            const R rl = R(1) / (d1 + R(2) * d0);
            const R rr = R(1) / (R(2) * d1 + d0);
            w0Left = d1 * rl;
            w1Left = R(2) * d0 * rl;
            w0Right = R(2) * d1 * rr;
            w1Right = d0 * rr;
        } else {
            const R a0Left = R(1) / d0;
            const R a1Right = R(1) / d1;
            const R a1Left = twice_reciprocal(d1, a1Right);
            const R a0Right = twice_reciprocal(d0, a0Left);
            w0Left = a0Left / (a0Left + a1Left);
            w1Left = a1Left / (a0Left + a1Left);
            w0Right = a0Right / (a0Right + a1Right);
            w1Right = a1Right / (a0Right + a1Right);
        }
        const R cl = R(3) * w0Left + w1Left;
        const R cr = R(3) * w1Right + w0Right;
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            const R um = f.at(v, -1);
            const R u0 = f.at(v, 0);
            const R up = f.at(v, 1);
            left[v] = R(0.5) * (w1Left * um + cl * u0 - w0Left * up);
            right[v] = R(0.5) * (w0Right * up + cr * u0 - w1Right * um);
        }
    } else if (RECON == RECON_WENO3) {
        // WENOCPU<3> (WENOCPU.cpp:34-187), WENOCoefficients<3>
        // (WENOCoefficients.hpp:52-66, WENOCoefficients.cpp:24-37): smoothness
        // of rho on the three ENO3 stencils, weights c_i / (beta_i + eps)^2
        // summed from i = 2 down, ENO3 candidate values combined per variable
        // (std::pow(x, 2) with its constant exponent is x*x)
        const R eps = R(1e-8);
        const R v0 = f.at(0, -2), v1 = f.at(0, -1), v2 = f.at(0, 0), v3 = f.at(0, 1), v4 = f.at(0, 2);
        const R c1312 = R(13.0 / 12.0);
        const R quarter = R(1 / 4.0);
        R q = v2 - R(2) * v3 + v4;
        R beta0 = c1312 * (q * q);
        q = R(3) * v2 - R(4) * v3 + v4;
        beta0 = beta0 + quarter * (q * q);
        q = v1 - R(2) * v2 + v3;
        R beta1 = c1312 * (q * q);
        q = v1 - v3;
        beta1 = beta1 + quarter * (q * q);
        q = v0 - R(2) * v1 + v2;
        R beta2 = c1312 * (q * q);
        q = v0 - R(4) * v1 + R(3) * v2;
        beta2 = beta2 + quarter * (q * q);
        const R cw0 = R(3.0 / 10.0), cw1 = R(3.0 / 5.0), cw2 = R(1.0 / 10.0);
        const R d2 = (beta2 + eps) * (beta2 + eps);
        const R d1 = (beta1 + eps) * (beta1 + eps);
        const R d0 = (beta0 + eps) * (beta0 + eps);
        R ar[3], al[3];
        ar[2] = cw2 / d2;
        al[2] = cw0 / d2;
        ar[1] = cw1 / d1;
        al[1] = cw1 / d1;
        ar[0] = cw0 / d0;
        al[0] = cw2 / d0;
        const R sr = ((R(0) + ar[2]) + ar[1]) + ar[0];
        const R sl = ((R(0) + al[2]) + al[1]) + al[0];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            R lw = R(0), rw = R(0);
#pragma unroll
            for (int shift = 0; shift < 3; ++shift) {
                R lv = R(0), rv = R(0);
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    const R value = f.at(v, j - shift);
                    lv += eno_coef<R, 3>(shift, j) * value;
                    rv += eno_coef<R, 3>(shift + 1, j) * value;
                }
                lw += lv * (al[shift] / sl);
                rw += rv * (ar[shift] / sr);
            }
            left[v] = lw;
            right[v] = rw;
        }
    } else if (RECON == RECON_WENOF2) {
        // WENOF2.hpp:37-121: WENO2 weights of rho, slopes in primitive variables
        constexpr int NSD = NV - 2;
        const R eps = R(1e-8);
        const R i0 = f.at(0, 0);
        const R dp = f.at(0, 1) - i0;
        const R dm = i0 - f.at(0, -1);
        const R b0 = dp * dp;
        const R b1 = dm * dm;
        const R d0 = R(3) * (eps + b0) * (eps + b0);
        const R d1 = R(3) * (eps + b1) * (eps + b1);
        R w0Left, w1Left, w0Right, w1Right;
        if constexpr (fast_recip<R>()) {
            // a0L = 1/d0, a1L = 2/d1, a0R = 2/d0, a1R = 1/d1 give w0L = d1/(d1 + 2 d0),
            // w1L = 2 d0/(d1 + 2 d0), w0R = 2 d1/(2 d1 + d0), w1R = d0/(2 d1 + d0)
            // (d stays finite in FP32 while neighbouring densities differ by < 1e9)
            const R rl = R(1) / (d1 + R(2) * d0);
            const R rr = R(1) / (R(2) * d1 + d0);
            w0Left = d1 * rl;
            w1Left = R(2) * d0 * rl;
            w0Right = R(2) * d1 * rr;
            w1Right = d0 * rr;
        } else {
            const R a0Left = R(1) / d0;
            const R a1Right = R(1) / d1;
            const R a1Left = twice_reciprocal(d1, a1Right);
            const R a0Right = twice_reciprocal(d0, a0Left);
            w0Left = a0Left / (a0Left + a1Left);
            w1Left = a1Left / (a0Left + a1Left);
            w0Right = a0Right / (a0Right + a1Right);
            w1Right = a1Right / (a0Right + a1Right);
        }
        R rho[3], u[3][NSD], p[3];
#pragma unroll
        for (int o = -1; o <= 1; ++o) {
            primitive_at<R, NSD>(f, o, gamma, rho[o + 1], u[o + 1], p[o + 1]);
        }
        wenof2_side<R, NSD, false>(w0Left, w1Left, gamma, rho, u, p, left);
        wenof2_side<R, NSD, true>(w0Right, w1Right, gamma, rho, u, p, right);
    } else if (RECON == RECON_MC || RECON == RECON_MM) {
        // MC.hpp:30-50 / MM.hpp:29-48, per variable
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            const R l = f.at(v, -1);
            const R m = f.at(v, 0);
            const R r = f.at(v, 1);
            R sigma;
            if (RECON == RECON_MC) {
                sigma = minmod3(R(2) * (r - m), (r - l) / R(2), R(2) * (m - l));
            } else {
                sigma = minmod2(r - m, m - l);
            }
            left[v] = m - sigma / R(2);
            right[v] = m + sigma / R(2);
        }
    } else {
        constexpr int ORDER = RECON == RECON_ENO2 ? 2 : (RECON == RECON_ENO3 ? 3 : 4);
        // undivided differences of rho at offsets -1..ORDER-2, level by level
        R dd[ORDER];
#pragma unroll
        for (int k = -1; k <= ORDER - 2; ++k) {
            dd[k + 1] = f.at(0, k + 1) - f.at(0, k);
        }
        int shift = 0;
#pragma unroll
        for (int level = 0; level < ORDER - 1; ++level) {
            if (level > 0) {
#pragma unroll
                for (int k = -1; k <= ORDER - 2 - level; ++k) {
                    dd[k + 1] = dd[k + 2] - dd[k + 1];
                }
            }
            if (fabs(dd[0]) < fabs(dd[1])) {
                shift++;
            }
        }
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            R lv = R(0), rv = R(0);
#pragma unroll
            for (int j = 0; j < ORDER; ++j) {
                const R value = f.dyn(v, j - shift);
                lv += eno_coef<R, ORDER>(shift, j) * value;
                rv += eno_coef<R, ORDER>(shift + 1, j) * value;
            }
            left[v] = lv;
            right[v] = rv;
        }
    }
}

// Stencil values from memory: variable v of the cell at `src` is v*vstride
// away, neighbours along the direction s apart.
template<class R, class I>
struct StridedFetch {
    const R* src;
    I vstride;
    I s;
    __device__ __forceinline__ R at(int v, int o) const { return src[v * vstride + o * s]; }
    __device__ __forceinline__ R dyn(int v, int o) const { return src[v * vstride + o * s]; }
};

template<class R, int NV, int RECON>
__device__ __forceinline__ void reconstruct(const R* src, int vstride, int s, R* left, R* right,
    R gamma) {
    StridedFetch<R, int> f{src, vstride, s};
    reconstruct_f<R, NV, RECON>(f, left, right, gamma);
}

} // namespace als
