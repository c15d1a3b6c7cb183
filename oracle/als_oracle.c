/*
 * CPU restatement of alsfvm's cell-update hot path (test oracle).
 *
 * TEST INFRASTRUCTURE ONLY -- see als_oracle.h.  Compiled with
 * -ffp-contract=off so that every a*b+c is two rounded operations, like the
 * reference CPU build; every expression keeps the reference's evaluation
 * order, which is cited beside it.
 */
#include "als_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define WENO_EPS 1e-8 /* WENOCoefficients.hpp:21 */

/* ---------------------------------------------------------------- Euler */

/* Conserved state plus the extra variables p and u of one cell
 * (AllVariables, Euler.hpp:96-101,204-211, 279-284). */
typedef struct {
    double rho, m[3], E;
    double p, u[3];
} state_t;

static void make_all(int nsd, double gamma, double rho, const double* m, double E,
    state_t* s) {
    double dot = 0.0;
    int k;
    s->rho = rho;
    s->E = E;
    for (k = 0; k < 3; ++k) {
        s->m[k] = k < nsd ? m[k] : 0.0;
    }
    /* vec dot: x*x + y*y + z*z, left to right (vec1/2/3.hpp dot) */
    dot = s->m[0] * s->m[0];
    if (nsd > 1) {
        dot = dot + s->m[1] * s->m[1];
    }
    if (nsd > 2) {
        dot = dot + s->m[2] * s->m[2];
    }
    /* ie = E - 0.5 * m.m / rho  (Euler.hpp:207) */
    {
        double ie = E - 0.5 * dot / rho;
        for (k = 0; k < 3; ++k) {
            s->u[k] = k < nsd ? s->m[k] / rho : 0.0; /* Euler.hpp:208 */
        }
        s->p = (gamma - 1) * ie; /* Euler.hpp:209 */
    }
}

/* Point flux in direction d (Euler.hpp:172-181). */
static void point_flux(int nsd, int d, const state_t* s, double* F) {
    int k;
    F[0] = s->m[d];
    for (k = 0; k < nsd; ++k) {
        F[1 + k] = s->m[k] * s->u[d];
    }
    F[1 + d] = F[1 + d] + s->p;
    F[1 + nsd] = (s->E + s->p) * s->u[d];
}

static void conserved_of(int nsd, const state_t* s, double* U) {
    int k;
    U[0] = s->rho;
    for (k = 0; k < nsd; ++k) {
        U[1 + k] = s->m[k];
    }
    U[1 + nsd] = s->E;
}

/* HLL, HLL.hpp:51-116. */
static double flux_hll(int nsd, int d, double gamma, const state_t* L, const state_t* R,
    double* F) {
    const int nv = nsd + 2;
    const double wl = sqrt(L->rho);
    const double wr = sqrt(R->rho);
    const double rho = (L->rho + R->rho) / 2;
    const double ud = (wl * L->u[d] + wr * R->u[d]) / (wl + wr);
    const double p = (L->p * wl + R->p * wr) / (wl + wr);
    const double cs = sqrt(gamma * p / rho);
    const double sL = fmin(L->u[d] - sqrt(gamma * L->p / L->rho), ud - cs);
    const double sR = fmax(R->u[d] + sqrt(gamma * R->p / R->rho), ud + cs);
    int k;
    if (sL == 0) {
        for (k = 0; k < nv; ++k) {
            F[k] = 0;
        }
    } else if (sL > 0) {
        point_flux(nsd, d, L, F);
    } else if (sR < 0) {
        point_flux(nsd, d, R, F);
    } else {
        double FL[5], FR[5], UL[5], UR[5];
        point_flux(nsd, d, L, FL);
        point_flux(nsd, d, R, FR);
        conserved_of(nsd, L, UL);
        conserved_of(nsd, R, UR);
        for (k = 0; k < nv; ++k) {
            F[k] = (sR * FL[k] - sL * FR[k] + sR * sL * (UR[k] - UL[k])) / (sR - sL);
        }
    }
    return fmax(fabs(sL), fabs(sR));
}

/* HLL3, HLL3.hpp:52-149. */
static double flux_hll3(int nsd, int d, double gamma, const state_t* L, const state_t* R,
    double* F) {
    const int nv = nsd + 2;
    const double wl = sqrt(L->rho);
    const double wr = sqrt(R->rho);
    const double rho = (L->rho + R->rho) / 2;
    const double ud = (wl * L->u[d] + wr * R->u[d]) / (wl + wr);
    const double p = (wl * L->p + wr * R->p) / (wl + wr);
    const double cfL = sqrt(gamma * L->p / L->rho);
    const double cfR = sqrt(gamma * R->p / R->rho);
    const double correct = 0.5 * fmax(0.0, L->u[d] - R->u[d]);
    const double cs = sqrt(gamma * p / rho);
    const double sL = fmin(L->u[d] + correct - cfL, ud - cs);
    const double sR = fmax(R->u[d] - correct + cfR, ud + cs);
    double FL[5], FR[5], us[3];
    int k;
    point_flux(nsd, d, L, FL);
    point_flux(nsd, d, R, FR);
    {
        const double pL = L->p, pR = R->p;
        const double udl = L->u[d] - sL;
        const double udr = R->u[d] - sR;
        const double aa = udr * R->rho - udl * L->rho;
        const double sm = (R->m[d] * udr - L->m[d] * udl + pR - pL) / aa;
        for (k = 0; k < nsd; ++k) {
            us[k] = (FR[1 + k] - FL[1 + k] - sR * R->m[k] + sL * L->m[k]) / aa;
        }
        us[d] = sm;
        if (sL == 0) {
            for (k = 0; k < nv; ++k) {
                F[k] = 0;
            }
        } else if (sL > 0) {
            for (k = 0; k < nv; ++k) {
                F[k] = FL[k];
            }
        } else if (sR < 0) {
            for (k = 0; k < nv; ++k) {
                F[k] = FR[k];
            }
        } else if (sm >= 0) {
            double mid[5], U[5];
            mid[0] = L->rho * udl / (sm - sL);
            for (k = 0; k < nsd; ++k) {
                mid[1 + k] = us[k] * mid[0];
            }
            {
                const double ps = pL + L->rho * (L->u[d] - sm) * udl;
                mid[1 + nsd] = (udl * L->E + pL * L->u[d] - ps * sm) / (sm - sL);
            }
            conserved_of(nsd, L, U);
            for (k = 0; k < nv; ++k) {
                F[k] = FL[k] + sL * (mid[k] - U[k]);
            }
        } else {
            double mid[5], U[5];
            mid[0] = R->rho * udr / (sm - sR);
            for (k = 0; k < nsd; ++k) {
                mid[1 + k] = us[k] * mid[0];
            }
            {
                const double ps = pR + R->rho * (R->u[d] - sm) * udr;
                mid[1 + nsd] = (udr * R->E + pR * R->u[d] - ps * sm) / (sm - sR);
            }
            conserved_of(nsd, R, U);
            for (k = 0; k < nv; ++k) {
                F[k] = FR[k] + sR * (mid[k] - U[k]);
            }
        }
    }
    return fmax(fabs(sL), fabs(sR));
}

/* Central, Central.hpp:39-56; wave speed Euler.hpp:251-258. */
static double flux_central(int nsd, int d, double gamma, const state_t* L,
    const state_t* R, double* F) {
    const int nv = nsd + 2;
    double FL[5], FR[5];
    int k;
    point_flux(nsd, d, L, FL);
    point_flux(nsd, d, R, FR);
    for (k = 0; k < nv; ++k) {
        F[k] = 0.5 * (FL[k] + FR[k]);
    }
    return fmax(fabs(L->u[d]) + sqrt(gamma * L->p / L->rho),
            fabs(R->u[d]) + sqrt(gamma * R->p / R->rho));
}

/* ---------------------------------------------------------------- TeCNO */

/* bar and ln of tecno_utils.hpp:22-38: the logarithmic mean is 0 when
 * either difference is 0; divLn (tecno_utils.hpp:42-50) gives 0 over it. */
static double tecno_bar(double a, double b) {
    return (a + b) / 2;
}

static double tecno_ln(double a, double b) {
    if (b - a == 0 || log(b) - log(a) == 0) {
        return 0;
    }
    return (b - a) / (log(b) - log(a));
}

static double tecno_div_ln(double a, double b, double F) {
    const double div = tecno_ln(a, b);
    return div == 0 ? 0 : F / div;
}

/* z = (sqrt(rho/p), sqrt(rho/p) u, sqrt(rho p)) from the primitive
 * variables u = m/rho, p = (gamma-1)(E - 0.5 m.m/rho) (Euler.hpp:290-320);
 * z has nsd+2 entries. */
static void tecno_z(int nsd, double gamma, const state_t* s, double* z) {
    double dot = s->m[0] * s->m[0];
    double p, q;
    int k;
    if (nsd > 1) {
        dot = dot + s->m[1] * s->m[1];
    }
    if (nsd > 2) {
        dot = dot + s->m[2] * s->m[2];
    }
    p = (gamma - 1) * (s->E - 0.5 * dot / s->rho);
    q = sqrt(s->rho / p);
    z[0] = q;
    for (k = 0; k < nsd; ++k) {
        z[1 + k] = (s->m[k] / s->rho) * q;
    }
    z[1 + nsd] = sqrt(s->rho * p);
}

/* Speeds of HLL3::computeHLLSpeeds (HLL3.hpp:120-160), as in flux_hll3. */
static double hll3_speed(int d, double gamma, const state_t* L, const state_t* R) {
    const double wl = sqrt(L->rho);
    const double wr = sqrt(R->rho);
    const double rho = (L->rho + R->rho) / 2;
    const double ud = (wl * L->u[d] + wr * R->u[d]) / (wl + wr);
    const double p = (wl * L->p + wr * R->p) / (wl + wr);
    const double cfL = sqrt(gamma * L->p / L->rho);
    const double cfR = sqrt(gamma * R->p / R->rho);
    const double correct = 0.5 * fmax(0.0, L->u[d] - R->u[d]);
    const double cs = sqrt(gamma * p / rho);
    const double sL = fmin(L->u[d] + correct - cfL, ud - cs);
    const double sR = fmax(R->u[d] - correct + cfR, ud + cs);
    return fmax(fabs(sL), fabs(sR));
}

/* Tecno1 (numflux/euler/Tecno1.hpp:51-180).  The reference writes the 2-D
 * formulas for all dimensions: in 3-D the z-momentum flux is 0, and along z
 * the flux keeps its zero initial value unless both states are equal. */
static double flux_tecno1(int nsd, int d, double gamma, const state_t* L, const state_t* R,
    double* F) {
    const int nv = nsd + 2;
    int same = L->rho == R->rho && L->E == R->E;
    int k;
    for (k = 0; k < nsd; ++k) {
        same = same && L->m[k] == R->m[k];
    }
    if (same) {
        point_flux(nsd, d, L, F);
    } else if (nsd == 3 && d == 2) {
        for (k = 0; k < nv; ++k) {
            F[k] = 0;
        }
    } else {
        double zl[5], zr[5], e;
        const int last = nsd + 1;
        tecno_z(nsd, gamma, L, zl);
        tecno_z(nsd, gamma, R, zr);
        F[0] = tecno_bar(zl[1 + d], zr[1 + d]) * tecno_ln(zl[last], zr[last]);
        for (k = 0; k < nsd; ++k) {
            if (nsd == 3 && k == 2) {
                F[1 + k] = 0;
            } else if (k == d) {
                F[1 + k] = tecno_bar(zl[last], zr[last]) / tecno_bar(zl[0], zr[0]) +
                    tecno_bar(zl[1 + d], zr[1 + d]) / tecno_bar(zl[0], zr[0]) * F[0];
            } else {
                F[1 + k] = tecno_bar(zl[1 + k], zr[1 + k]) / tecno_bar(zl[0], zr[0]) * F[0];
            }
        }
        e = (gamma + 1) / (gamma - 1) * tecno_div_ln(zl[0], zr[0], F[0]) +
            tecno_bar(zl[1], zr[1]) * F[1];
        if (nsd > 1) {
            e = e + tecno_bar(zl[2], zr[2]) * F[2];
        }
        F[last] = 1.0 / (2 * tecno_bar(zl[0], zr[0])) * e;
    }
    return hll3_speed(d, gamma, L, R);
}

/* TecnoCombined4 / TecnoCombined6 (TecnoCombined4.hpp:40-60,
 * TecnoCombined6.hpp:40-65) at the face between cells c and c+s of `in`.
 * TecnoCombined6's stencil {-2, -1, 0, 1, 2, 3} is held in an ivec6 whose
 * constructor stores 0 for the sixth entry (alsutils/vec6.hpp:36-39), so
 * its "u_{i+3}" is u_i and the last term is F(u_i, u_i), the point flux. */
static double flux_tecno_stencil(const orc_config* cfg, int d, const double* in, long plane,
    long c, long s, double* F) {
    const int nsd = cfg->dim;
    const int nv = nsd + 2;
    double w = 0;
    double f[6][5];
    /* pairs (a, b): F(u_{c+a}, u_{c+b}) */
    static const int pairs[6][2] = {{0, 1}, {-1, 1}, {0, 2}, {-2, 1}, {-1, 2}, {0, 0}};
    const int np = cfg->flux == ORC_FLUX_TECNO4 ? 3 : 6;
    int k, q;
    for (q = 0; q < np; ++q) {
        state_t A, B;
        double ua[5], ub[5];
        int v;
        for (v = 0; v < nv; ++v) {
            ua[v] = in[v * plane + c + pairs[q][0] * s];
            ub[v] = in[v * plane + c + pairs[q][1] * s];
        }
        make_all(nsd, cfg->gamma, ua[0], ua + 1, ua[1 + nsd], &A);
        make_all(nsd, cfg->gamma, ub[0], ub + 1, ub[1 + nsd], &B);
        w = fmax(w, flux_tecno1(nsd, d, cfg->gamma, &A, &B, f[q]));
    }
    for (k = 0; k < nv; ++k) {
        if (np == 3) {
            F[k] = 4.0 / 3.0 * f[0][k] - 1.0 / 6.0 * (f[1][k] + f[2][k]);
        } else {
            F[k] = (3.0 / 2.0 * f[0][k] - 3.0 / 10.0 * (f[1][k] + f[2][k])) +
                1.0 / 30.0 * ((f[3][k] + f[4][k]) + f[5][k]);
        }
    }
    return w;
}

/* -------------------------------------------------------------- helpers */

int orc_ghost_cells(int flux, int recon) {
    int rg = 1;
    /* stencil size - 1: 3 for tecno4, 5 for tecno6, else 1 (numflux_util.hpp:52-60) */
    const int fg = flux == ORC_FLUX_TECNO4 ? 3 : (flux == ORC_FLUX_TECNO6 ? 5 : 1);
    if (flux < ORC_FLUX_HLL || flux > ORC_FLUX_TECNO6) {
        return -1;
    }
    switch (recon) {
    case ORC_RECON_NONE: rg = 1; break;
    case ORC_RECON_WENO2: rg = 2; break;
    case ORC_RECON_ENO2: rg = 2; break;
    case ORC_RECON_ENO3: rg = 3; break;
    case ORC_RECON_ENO4: rg = 4; break;
    case ORC_RECON_MC: rg = 2; break;
    case ORC_RECON_MM: rg = 2; break;
    case ORC_RECON_WENOF2: rg = 2; break;
    case ORC_RECON_WENO3: rg = 3; break;
    default: return -1;
    }
    return rg > fg ? rg : fg;
}

int orc_configure(orc_config* cfg, int dim, const int* n, const double* lower,
    const double* upper, int flux, int recon, int integrator, int bc, double gamma) {
    int d;
    if (dim < 1 || dim > 3) {
        return -1;
    }
    memset(cfg, 0, sizeof(*cfg));
    cfg->diffusion = -1;
    cfg->dim = dim;
    for (d = 0; d < 3; ++d) {
        cfg->n[d] = d < dim ? n[d] : 1;
    }
    cfg->g = orc_ghost_cells(flux, recon);
    if (cfg->g < 0) {
        return -1;
    }
    cfg->gamma = gamma;
    cfg->flux = flux;
    cfg->recon = recon;
    cfg->integrator = integrator;
    cfg->bc = bc;
    for (d = 0; d < 3; ++d) {
        /* Grid.cpp:30-38: (top-origin)/n, and 1 for directions with one cell */
        cfg->dx[d] = (upper[d] - lower[d]) / (double)cfg->n[d];
        if (d > 0 && cfg->n[d] == 1) {
            cfg->dx[d] = 1;
        }
    }
    return 0;
}

static void padded(const orc_config* cfg, int* N) {
    int d;
    for (d = 0; d < 3; ++d) {
        N[d] = cfg->n[d] + (d < cfg->dim ? 2 * cfg->g : 0);
    }
}

long orc_plane_size(const orc_config* cfg) {
    int N[3];
    padded(cfg, N);
    return (long)N[0] * N[1] * N[2];
}

static long idx3(const int* N, int x, int y, int z) {
    return ((long)z * N[1] + y) * N[0] + x;
}

/* ------------------------------------------------------------- boundary */

void orc_fill_ghosts(const orc_config* cfg, double* planes, int nvar) {
    int N[3];
    const int g = cfg->g;
    const long plane = orc_plane_size(cfg);
    int var, d, side;
    padded(cfg, N);
    for (var = 0; var < nvar; ++var) {
        double* u = planes + var * plane;
        for (d = 0; d < cfg->dim; ++d) {
            for (side = 0; side < 2; ++side) {
                /* the side loop covers the full transverse extent, ghosts included */
                int x, y, z, k;
                const int n = cfg->n[d];
                const int first = side == 0 ? g : N[d] - g - 1;
                for (z = 0; z < (d == 2 ? 1 : N[2]); ++z) {
                    for (y = 0; y < (d == 1 ? 1 : N[1]); ++y) {
                        for (x = 0; x < (d == 0 ? 1 : N[0]); ++x) {
                            int c[3];
                            c[0] = x;
                            c[1] = y;
                            c[2] = z;
                            for (k = 1; k <= g; ++k) {
                                int dst[3], src[3];
                                memcpy(dst, c, sizeof(dst));
                                memcpy(src, c, sizeof(src));
                                if (cfg->bc == ORC_BC_NEUMANN) {
                                    /* mirror: ghost[g-k] = U[g+k-1], ghost[N-g-1+k] = U[N-g-k] */
                                    dst[d] = side == 0 ? first - k : first + k;
                                    src[d] = side == 0 ? first + (k - 1) : first - (k - 1);
                                } else {
                                    /* periodic: ghost[g-k] = U[g-k+n], ghost[N-g-1+k] = U[N-g-1+k-n] */
                                    dst[d] = side == 0 ? first - k : first + k;
                                    src[d] = side == 0 ? first + (n - k) : first - (n - k);
                                }
                                u[idx3(N, dst[0], dst[1], dst[2])] =
                                    u[idx3(N, src[0], src[1], src[2])];
                            }
                        }
                    }
                }
            }
        }
    }
}

/* ------------------------------------------------------- reconstruction */

static const double eno2c[3][2] = {
    {3.0 / 2.0, -1.0 / 2.0},
    {1.0 / 2.0, 1.0 / 2.0},
    {-1.0 / 2.0, 3.0 / 2.0}
};
static const double eno3c[4][3] = {
    {11.0 / 6.0, -7.0 / 6.0, 1.0 / 3.0},
    {1.0 / 3.0, 5.0 / 6.0, -1.0 / 6.0},
    {-1.0 / 6.0, 5.0 / 6.0, 1.0 / 3.0},
    {1.0 / 3.0, -7.0 / 6.0, 11.0 / 6.0}
};
static const double eno4c[5][4] = {
    {25.0 / 12.0, -23.0 / 12.0, 13.0 / 12.0, -1.0 / 4.0},
    {1.0 / 4.0, 13.0 / 12.0, -5.0 / 12.0, 1.0 / 12.0},
    {-1.0 / 12.0, 7.0 / 12.0, 7.0 / 12.0, -1.0 / 12.0},
    {1.0 / 12.0, -5.0 / 12.0, 13.0 / 12.0, 1.0 / 4.0},
    {-1.0 / 4.0, 13.0 / 12.0, -23.0 / 12.0, 25.0 / 12.0}
};

static double eno_coef(int order, int r, int j) {
    switch (order) {
    case 2: return eno2c[r][j];
    case 3: return eno3c[r][j];
    default: return eno4c[r][j];
    }
}

static double sign_of(double a) {
    return a > 0 ? 1.0 : (a == 0 ? 0.0 : -1.0);
}

static double minmod2(double a, double b) {
    if (sign_of(a) == sign_of(b)) {
        return sign_of(a) * fmin(fabs(a), fabs(b));
    }
    return 0;
}

static double minmod3(double a, double b, double c) {
    if (sign_of(a) == sign_of(b) && sign_of(b) == sign_of(c)) {
        return sign_of(a) * fmin(fabs(a), fmin(fabs(b), fabs(c)));
    }
    return 0;
}

/* Reconstructs cell c (index into the planes) along stride s.
 * left/right receive nvar values. */
static void reconstruct_cell(const orc_config* cfg, const double* in, long plane,
    long c, long s, int nvar, double* left, double* right) {
    int var;
    if (cfg->recon == ORC_RECON_NONE) {
        for (var = 0; var < nvar; ++var) {
            left[var] = in[var * plane + c];
            right[var] = in[var * plane + c];
        }
    } else if (cfg->recon == ORC_RECON_WENO2) {
        /* WENO2.hpp:37-69; the indicator is rho (Euler.hpp:286-288) */
        const double i0 = in[c];
        const double b0 = (in[c + s] - i0) * (in[c + s] - i0);
        const double b1 = (i0 - in[c - s]) * (i0 - in[c - s]);
        const double a0Left = 1 / (3 * (WENO_EPS + b0) * (WENO_EPS + b0));
        const double a1Left = 2 / (3 * (WENO_EPS + b1) * (WENO_EPS + b1));
        const double w0Left = a0Left / (a0Left + a1Left);
        const double w1Left = a1Left / (a0Left + a1Left);
        const double a0Right = 2 / (3 * (WENO_EPS + b0) * (WENO_EPS + b0));
        const double a1Right = 1 / (3 * (WENO_EPS + b1) * (WENO_EPS + b1));
        const double w0Right = a0Right / (a0Right + a1Right);
        const double w1Right = a1Right / (a0Right + a1Right);
        for (var = 0; var < nvar; ++var) {
            const double um = in[var * plane + c - s];
            const double u0 = in[var * plane + c];
            const double up = in[var * plane + c + s];
            left[var] = 0.5 * (w1Left * um + (3 * w0Left + w1Left) * u0 - w0Left * up);
            right[var] = 0.5 * (w0Right * up + (3 * w1Right + w0Right) * u0 - w1Right * um);
        }
    } else if (cfg->recon == ORC_RECON_WENO3) {
        /* WENOCPU<3> (WENOCPU.cpp:34-187) with WENOCoefficients<3>
         * (WENOCoefficients.hpp:52-66, WENOCoefficients.cpp:24-37); the
         * reference's std::pow(x, 2) has a constant exponent and is x*x */
        static const double c3[3] = {3.0 / 10.0, 3.0 / 5.0, 1.0 / 10.0};
        const double eps = 1e-8;
        double V[5], beta[3], al[3], ar[3], sl = 0.0, sr = 0.0, q;
        int i, shift, j;
        for (i = -2; i <= 2; ++i) {
            V[i + 2] = in[c + i * s];
        }
        q = V[2] - 2 * V[3] + V[4];
        beta[0] = 13.0 / 12.0 * (q * q);
        q = 3 * V[2] - 4 * V[3] + V[4];
        beta[0] = beta[0] + 1 / 4.0 * (q * q);
        q = V[1] - 2 * V[2] + V[3];
        beta[1] = 13.0 / 12.0 * (q * q);
        q = V[1] - V[3];
        beta[1] = beta[1] + 1 / 4.0 * (q * q);
        q = V[0] - 2 * V[1] + V[2];
        beta[2] = 13.0 / 12.0 * (q * q);
        q = V[0] - 4 * V[1] + 3 * V[2];
        beta[2] = beta[2] + 1 / 4.0 * (q * q);
        for (i = 2; i >= 0; --i) {
            const double d = (beta[i] + eps) * (beta[i] + eps);
            ar[i] = c3[i] / d;
            sr += ar[i];
            al[i] = c3[2 - i] / d;
            sl += al[i];
        }
        for (var = 0; var < nvar; ++var) {
            double lw = 0.0, rw = 0.0;
            for (shift = 0; shift < 3; ++shift) {
                double lv = 0.0, rv = 0.0;
                for (j = 0; j < 3; ++j) {
                    const double value = in[var * plane + c - (long)(shift - j) * s];
                    lv += eno_coef(3, shift, j) * value;
                    rv += eno_coef(3, shift + 1, j) * value;
                }
                lw += lv * (al[shift] / sl);
                rw += rv * (ar[shift] / sr);
            }
            left[var] = lw;
            right[var] = rw;
        }
    } else if (cfg->recon == ORC_RECON_WENOF2) {
        /* WENOF2.hpp:37-121: weights as WENO2, slopes of the primitive
         * variables (Euler.hpp:290-297) bounded, limited, back to conserved
         * variables (Euler.hpp:236-245) */
        const int nsd = nvar - 2;
        const double BOUND = 1.9;
        const double gm1 = cfg->gamma - 1;
        const double i0 = in[c];
        const double b0 = (in[c + s] - i0) * (in[c + s] - i0);
        const double b1 = (i0 - in[c - s]) * (i0 - in[c - s]);
        const double a0Left = 1 / (3 * (WENO_EPS + b0) * (WENO_EPS + b0));
        const double a1Left = 2 / (3 * (WENO_EPS + b1) * (WENO_EPS + b1));
        const double w0Left = a0Left / (a0Left + a1Left);
        const double w1Left = a1Left / (a0Left + a1Left);
        const double a0Right = 2 / (3 * (WENO_EPS + b0) * (WENO_EPS + b0));
        const double a1Right = 1 / (3 * (WENO_EPS + b1) * (WENO_EPS + b1));
        const double w0Right = a0Right / (a0Right + a1Right);
        const double w1Right = a1Right / (a0Right + a1Right);
        double rho[3], u[3][3], p[3];
        int o, k, side;
        for (o = 0; o < 3; ++o) {
            const long cc = c + (o - 1) * s;
            double dot = in[plane + cc] * in[plane + cc];
            for (k = 1; k < nsd; ++k) {
                dot = dot + in[(1 + k) * plane + cc] * in[(1 + k) * plane + cc];
            }
            rho[o] = in[cc];
            for (k = 0; k < nsd; ++k) {
                u[o][k] = in[(1 + k) * plane + cc] / rho[o];
            }
            p[o] = gm1 * (in[(nsd + 1) * plane + cc] - 0.5 * dot / rho[o]);
        }
        for (side = 0; side < 2; ++side) {
            const double w0 = side == 0 ? w0Left : w0Right;
            const double w1 = side == 0 ? w1Left : w1Right;
            double* out = side == 0 ? left : right;
            double dr = w1 * (rho[1] - rho[0]) + w0 * (rho[2] - rho[1]);
            double du[3], dp, dudu, umdu, LL, Rr, a, pr, pu[3], pp, dot;
            for (k = 0; k < nsd; ++k) {
                du[k] = w1 * (u[1][k] - u[0][k]) + w0 * (u[2][k] - u[1][k]);
            }
            dp = w1 * (p[1] - p[0]) + w0 * (p[2] - p[1]);
            dr = fmax(-BOUND * rho[1], fmin(BOUND * rho[1], dr));
            dp = fmax(-BOUND * p[1], fmin(BOUND * p[1], dp));
            dudu = du[0] * du[0];
            umdu = u[1][0] * du[0];
            for (k = 1; k < nsd; ++k) {
                dudu = dudu + du[k] * du[k];
                umdu = umdu + u[1][k] * du[k];
            }
            LL = 0.125 * rho[1] * dudu - 0.5 * fmin(0.0, dr * umdu) + 0.5 * dr * dr * dudu / rho[1];
            Rr = p[1] / (cfg->gamma - 1);
            a = 0.5 * sqrt(Rr / fmax(Rr, LL));
            pr = side == 0 ? rho[1] - a * dr : rho[1] + a * dr;
            pp = side == 0 ? p[1] - a * dp : p[1] + a * dp;
            dot = 0;
            for (k = 0; k < nsd; ++k) {
                pu[k] = side == 0 ? u[1][k] - a * du[k] : u[1][k] + a * du[k];
                dot = k == 0 ? pu[0] * pu[0] : dot + pu[k] * pu[k];
            }
            out[0] = pr;
            for (k = 0; k < nsd; ++k) {
                out[1 + k] = pr * pu[k];
            }
            out[nsd + 1] = pp / (cfg->gamma - 1) + 0.5 * pr * dot;
        }
    } else if (cfg->recon == ORC_RECON_MC || cfg->recon == ORC_RECON_MM) {
        /* MC.hpp:30-50 / MM.hpp:29-48 with minmod.hpp, sign.hpp, per variable */
        for (var = 0; var < nvar; ++var) {
            const double l = in[var * plane + c - s];
            const double m = in[var * plane + c];
            const double r = in[var * plane + c + s];
            const double sigma = cfg->recon == ORC_RECON_MC
                ? minmod3(2 * (r - m), (r - l) / 2, 2 * (m - l))
                : minmod2(r - m, m - l);
            left[var] = m - sigma / 2;
            right[var] = m + sigma / 2;
        }
    } else {
        /* ENOCPU.cpp:140-180.  Level-l undivided differences of rho:
         * DD0[i] = rho[i+1]-rho[i], DDl[i] = DD(l-1)[i+1]-DD(l-1)[i]
         * (ENOCPU.cpp:205-267); compare |DD[i-1]| < |DD[i]| per level. */
        const int order = cfg->recon == ORC_RECON_ENO2 ? 2 : (cfg->recon == ORC_RECON_ENO3 ? 3 : 4);
        int shift = 0, level, j, k;
        double dd[5]; /* dd[k+1] = level difference at offset k*s from c, k = -1..3 */
        for (k = -1; k <= order - 2; ++k) {
            dd[k + 1] = in[c + (k + 1) * s] - in[c + k * s];
        }
        for (level = 0; level < order - 1; ++level) {
            if (level > 0) {
                for (k = -1; k <= order - 2 - level; ++k) {
                    dd[k + 1] = dd[k + 2] - dd[k + 1];
                }
            }
            if (fabs(dd[0]) < fabs(dd[1])) {
                shift++;
            }
        }
        for (var = 0; var < nvar; ++var) {
            double lv = 0.0, rv = 0.0;
            for (j = 0; j < order; ++j) {
                const double value = in[var * plane + c - (long)(shift - j) * s];
                lv += eno_coef(order, shift, j) * value;
                rv += eno_coef(order, shift + 1, j) * value;
            }
            left[var] = lv;
            right[var] = rv;
        }
    }
}

void orc_reconstruct(const orc_config* cfg, int dir, const double* in, double* left,
    double* right) {
    int N[3];
    const int g = cfg->g;
    const int nvar = cfg->dim + 2;
    const long plane = orc_plane_size(cfg);
    long s;
    int lo[3], hi[3], d, x, y, z, var;
    padded(cfg, N);
    if (cfg->recon == ORC_RECON_NONE) {
        /* NoReconstruction copies every cell, ghosts included (NoReconstruction.cpp:51-61) */
        memcpy(left, in, sizeof(double) * (size_t)nvar * (size_t)plane);
        memcpy(right, in, sizeof(double) * (size_t)nvar * (size_t)plane);
        return;
    }
    s = dir == 0 ? 1 : (dir == 1 ? N[0] : (long)N[0] * N[1]);
    for (d = 0; d < 3; ++d) {
        const int gd = d < cfg->dim ? g : 0;
        lo[d] = gd - (d == dir ? 1 : 0);
        hi[d] = N[d] - gd + (d == dir ? 1 : 0);
        if (cfg->recon == ORC_RECON_WENO3 && d != dir) {
            /* WENOCPU.cpp:100-106: every cell across the direction, ghosts included */
            lo[d] = 0;
            hi[d] = N[d];
        }
    }
    for (z = lo[2]; z < hi[2]; ++z) {
        for (y = lo[1]; y < hi[1]; ++y) {
            for (x = lo[0]; x < hi[0]; ++x) {
                double l[5], r[5];
                const long c = idx3(N, x, y, z);
                reconstruct_cell(cfg, in, plane, c, s, nvar, l, r);
                for (var = 0; var < nvar; ++var) {
                    left[var * plane + c] = l[var];
                    right[var * plane + c] = r[var];
                }
            }
        }
    }
}

/* ------------------------------------------------------------ net flux */

static double face_flux(const orc_config* cfg, int d, const double* ul, const double* ur,
    double* F) {
    const int nsd = cfg->dim;
    state_t L, R;
    make_all(nsd, cfg->gamma, ul[0], ul + 1, ul[1 + nsd], &L);
    make_all(nsd, cfg->gamma, ur[0], ur + 1, ur[1 + nsd], &R);
    switch (cfg->flux) {
    case ORC_FLUX_HLL: return flux_hll(nsd, d, cfg->gamma, &L, &R, F);
    case ORC_FLUX_HLL3: return flux_hll3(nsd, d, cfg->gamma, &L, &R, F);
    case ORC_FLUX_TECNO1: return flux_tecno1(nsd, d, cfg->gamma, &L, &R, F);
    default: return flux_central(nsd, d, cfg->gamma, &L, &R, F);
    }
}

void orc_net_flux(const orc_config* cfg, const double* in, double* out, double ws[3]) {
    const int stencil = cfg->flux == ORC_FLUX_TECNO4 || cfg->flux == ORC_FLUX_TECNO6;
    int N[3];
    const int g = cfg->g;
    const int nvar = cfg->dim + 2;
    const long plane = orc_plane_size(cfg);
    int d, x, y, z, var;
    padded(cfg, N);
    /* makeZero over interior cells (NumericalFluxCPU.cpp:122-146) */
    for (z = (cfg->dim > 2 ? g : 0); z < N[2] - (cfg->dim > 2 ? g : 0); ++z) {
        for (y = (cfg->dim > 1 ? g : 0); y < N[1] - (cfg->dim > 1 ? g : 0); ++y) {
            for (x = g; x < N[0] - g; ++x) {
                for (var = 0; var < nvar; ++var) {
                    out[var * plane + idx3(N, x, y, z)] = 0;
                }
            }
        }
    }
    ws[0] = ws[1] = ws[2] = 0;
    if (stencil && cfg->recon != ORC_RECON_NONE) {
        return; /* stencil fluxes are restated for reconstruction none only */
    }
    for (d = 0; d < cfg->dim; ++d) {
        const long s = d == 0 ? 1 : (d == 1 ? N[0] : (long)N[0] * N[1]);
        const int len = N[d];
        int lo[3], hi[3];
        double wmax = 0;
        double* rec = (double*)malloc(sizeof(double) * 2 * nvar * (size_t)len);
        double* flux = (double*)malloc(sizeof(double) * nvar * (size_t)len);
        for (x = 0; x < 3; ++x) {
            const int gx = x < cfg->dim ? g : 0;
            lo[x] = gx;
            hi[x] = N[x] - gx;
        }
        lo[d] = 0;
        hi[d] = 1;
        for (z = lo[2]; z < hi[2]; ++z) {
            for (y = lo[1]; y < hi[1]; ++y) {
                for (x = lo[0]; x < hi[0]; ++x) {
                    /* one line along d through (x,y,z) */
                    const long base = idx3(N, x, y, z);
                    int i;
                    for (i = g - 1; i < len - g + 1; ++i) {
                        reconstruct_cell(cfg, in, plane, base + i * s, s, nvar,
                            rec + (size_t)i * 2 * nvar, rec + (size_t)i * 2 * nvar + nvar);
                    }
                    /* faces i|i+1 for i in [g-1, len-g): U- = right[i], U+ = left[i+1]
                     * (numflux_util.hpp:62-92); temp = -F (NumericalFluxCPU.cpp:92) */
                    for (i = g - 1; i < len - g; ++i) {
                        const double* ul = rec + (size_t)i * 2 * nvar + nvar;
                        const double* ur = rec + (size_t)(i + 1) * 2 * nvar;
                        /* stencil fluxes read the "left" volume, a copy of
                         * the cells under reconstruction none
                         * (numflux_util.hpp:94-116) */
                        const double w = stencil
                            ? flux_tecno_stencil(cfg, d, in, plane, base + i * s, s,
                                  flux + (size_t)i * nvar)
                            : face_flux(cfg, d, ul, ur, flux + (size_t)i * nvar);
                        if (wmax < w) { /* std::max(waveSpeedComputed, local) */
                            wmax = w;
                        }
                    }
                    /* out[i] += (-F_{i+1/2}) + (-(-F_{i-1/2})) (NumericalFluxCPU.cpp:100-117) */
                    for (i = g; i < len - g; ++i) {
                        for (var = 0; var < nvar; ++var) {
                            const double tr = -flux[(size_t)i * nvar + var];
                            const double tl = -flux[(size_t)(i - 1) * nvar + var];
                            out[var * plane + base + i * s] += tr + (-tl);
                        }
                    }
                }
            }
        }
        ws[d] = wmax;
        free(rec);
        free(flux);
    }
}

/* ---------------------------------------------------------- constraints */

int orc_obeys_constraints(const orc_config* cfg, const double* planes) {
    const int nsd = cfg->dim;
    const int nvar = nsd + 2;
    const long plane = orc_plane_size(cfg);
    long c;
    int var;
    for (c = 0; c < plane; ++c) {
        double U[5];
        state_t s;
        for (var = 0; var < nvar; ++var) {
            U[var] = planes[var * plane + c];
            if (isnan(U[var]) || isinf(U[var])) {
                return 0;
            }
        }
        make_all(nsd, cfg->gamma, U[0], U + 1, U[1 + nsd], &s);
        for (var = 0; var < nsd; ++var) {
            if (isnan(s.u[var]) || isinf(s.u[var])) {
                return 0;
            }
        }
        if (isnan(s.p) || isinf(s.p)) {
            return 0;
        }
        if (!(s.rho > 0) || !(s.p > 0)) {
            return 0;
        }
    }
    return 1;
}

/* ------------------------------------------------------------ time loop */

int orc_simulate(const orc_config* cfg, double cfl, double end_time, long max_steps,
    double* planes, double* dts, long dts_capacity, long* steps_out, double* t_out) {
    const int nvar = cfg->dim + 2;
    const long plane = orc_plane_size(cfg);
    const size_t bytes = sizeof(double) * (size_t)nvar * (size_t)plane;
    const int substeps = cfg->integrator + 1;
    double* vol[5];
    double* diff_state = NULL;
    double t = 0;
    long steps = 0, i;
    int s, status = 0, d;
    for (d = 0; d < cfg->dim; ++d) {
        if (cfg->n[d] < 2 * cfg->g) {
            return -1;
        }
    }
    for (s = 0; s <= substeps; ++s) {
        vol[s] = (double*)calloc(1, bytes);
    }
    memcpy(vol[0], planes, bytes);
    orc_fill_ghosts(cfg, vol[0], nvar);
    if (cfg->diffusion >= 0) {
        /* the operator's work arrays live as long as the simulator */
        const long vol4 = 4L * nvar * plane;
        diff_state = (double*)calloc((size_t)(vol4 + 3 * plane), sizeof(double));
        for (i = 0; i < vol4; ++i) {
            diff_state[i] = 42.0;
        }
    }
    while (t < end_time && steps < max_steps) {
        double dt = 0;
        for (s = 0; s < substeps; ++s) {
            double ws[3];
            double* out = vol[s + 1];
            const double* Us = vol[s];
            const double* U0 = vol[0];
            double c;
            orc_net_flux(cfg, Us, out, ws);
            if (diff_state) {
                orc_diffusion_apply(cfg, cfg->diffusion, cfg->diffusion_recon, diff_state, Us, out);
            }
            if (s == 0) {
                /* Integrator.cpp:20-46 then the end-time clamp */
                double total = 0;
                for (d = 0; d < 3; ++d) {
                    if (cfg->dx[d] == 0) {
                        continue;
                    }
                    total += ws[d] / cfg->dx[d];
                }
                dt = cfl / total;
                dt = (end_time - t < dt) ? end_time - t : dt;
            }
            c = dt / cfg->dx[0];
            /* the Volume operations run over every cell; ghosts are refilled below */
            if (cfg->integrator == ORC_INT_RK4) {
                /* RungeKutta4.cpp:66-87; the last stage is
                 * addLinearCombination (HostMemory.cpp:261-280) */
                const double a1 = (1.0 / 6.0) * c;
                for (i = 0; i < nvar * plane; ++i) {
                    double v = out[i];
                    if (s < 3) {
                        v *= c;
                        if (s < 2) {
                            v *= 0.5;
                        }
                        v += U0[i];
                    } else {
                        v = a1 * v + 1.0 / 3.0 * vol[1][i] + 2.0 / 3.0 * vol[2][i] +
                            1.0 / 3.0 * vol[3][i] + -1.0 / 3.0 * U0[i];
                    }
                    out[i] = v;
                }
                orc_fill_ghosts(cfg, out, nvar);
                continue;
            }
            for (i = 0; i < nvar * plane; ++i) {
                double v = out[i];
                v *= c;
                v += Us[i];
                if (cfg->integrator == ORC_INT_RK3 && s == 1) {
                    v *= 1. / 3.;
                    v += U0[i];
                    v *= 3. / 4.;
                } else if (cfg->integrator == ORC_INT_RK3 && s == 2) {
                    v *= 2;
                    v += U0[i];
                    v *= 1. / 3.;
                } else if (cfg->integrator == ORC_INT_RK2 && s == 1) {
                    v += U0[i];
                    v *= 0.5;
                }
                out[i] = v;
            }
            orc_fill_ghosts(cfg, out, nvar);
        }
        {
            double* tmp = vol[0];
            vol[0] = vol[substeps];
            vol[substeps] = tmp;
        }
        t += dt;
        if (dts && steps < dts_capacity) {
            dts[steps] = dt;
        }
        ++steps;
        if (!orc_obeys_constraints(cfg, vol[0])) {
            status = 1;
            break;
        }
    }
    memcpy(planes, vol[0], bytes);
    for (s = 0; s <= substeps; ++s) {
        free(vol[s]);
    }
    free(diff_state);
    if (steps_out) {
        *steps_out = steps;
    }
    if (t_out) {
        *t_out = t;
    }
    return status;
}

/* ----------------------------------------------------------- statistics */

void orc_meanvar(long count, long samples, const double* states, double* mean, double* var) {
    /* a run-time exponent, as in HostMemory::addPower, so the call is not folded to u*u */
    volatile double two = 2.0;
    long i, k;
    for (i = 0; i < count; ++i) {
        mean[i] = 0;
        var[i] = 0;
    }
    for (k = 0; k < samples; ++k) {
        for (i = 0; i < count; ++i) {
            const double u = states[k * count + i];
            mean[i] += u;
            var[i] += pow(u, two);
        }
    }
    for (i = 0; i < count; ++i) {
        mean[i] /= (double)samples;
        var[i] /= (double)samples;
        var[i] -= pow(mean[i], two);
    }
}

/* ------------------------------------------------------ structure functions */

/* ValueAtBoundary<PERIODIC/NEUMANN>::getValueAtBoundary, ValueAtBoundary.hpp:20-110 */
static double value_at(const double* plane, const int* n, const int* gh, const int* N, int bc,
    int x, int y, int z) {
    int pos[3] = {x, y, z};
    int d;
    for (d = 0; d < 3; ++d) {
        if (bc == ORC_BC_PERIODIC) {
            while (pos[d] < 0) {
                pos[d] += n[d];
            }
            pos[d] = pos[d] % n[d];
        } else {
            if (pos[d] > n[d] - 1) {
                pos[d] = n[d] - 1;
            }
            if (pos[d] < 0) {
                pos[d] = 0;
            }
        }
        pos[d] += gh[d];
    }
    return plane[((long)pos[2] * N[1] + pos[1]) * N[0] + pos[0]];
}

/* FastPower<p> (alsutils/math/FastPower.hpp): x * FastPower<p-1>(x); PowPower: pow */
static double structure_power(double x, double p) {
    if (p == 1.0) {
        return x;
    } else if (p == 2.0) {
        return x * x;
    } else if (p == 3.0) {
        return x * (x * x);
    } else if (p == 4.0) {
        return x * (x * (x * x));
    } else if (p == 5.0) {
        return x * (x * (x * (x * x)));
    }
    return pow(x, p);
}

static void structure_geometry(int dim, const int* n, int g, int* nn, int* gh, int* N) {
    int d;
    for (d = 0; d < 3; ++d) {
        nn[d] = d < dim ? n[d] : 1;
        gh[d] = d < dim ? g : 0;
        N[d] = nn[d] + 2 * gh[d];
    }
}

void orc_structure_cube(int dim, const int* n, int g, int bc, int nvar, int H, double p,
    const double* planes, double* out) {
    int nn[3], gh[3], N[3];
    long plane;
    int v, i, j, k, h, d, side, x, y, z;
    structure_geometry(dim, n, g, nn, gh, N);
    plane = (long)N[0] * N[1] * N[2];
    for (v = 0; v < nvar * H; ++v) {
        out[v] = 0;
    }
    for (v = 0; v < nvar; ++v) {
        const double* u_plane = planes + v * plane;
        double* o = out + (long)v * H;
        for (k = 0; k < nn[2]; ++k) {
            for (j = 0; j < nn[1]; ++j) {
                for (i = 0; i < nn[0]; ++i) {
                    const double u = u_plane[((long)(k + gh[2]) * N[1] + j + gh[1]) * N[0] + i + gh[0]];
                    for (h = 1; h < H; ++h) {
                        /* forEachPointInComputeStructureCube, structure_common.hpp:39-104 */
                        for (d = 0; d < dim; ++d) {
                            for (side = 0; side < 2; ++side) {
                                const int zDir = d == 2, yDir = d == 1, xDir = d == 0;
                                const int zStart = zDir ? (side == 0 ? k - h : k + h) : (dim > 2 ? k - h : 0);
                                const int zEnd = zDir ? zStart + 1 : (dim > 2 ? k + h + 1 : 1);
                                const int yStart = yDir ? (side == 0 ? j - h : j + h)
                                                        : (dim >= 2 ? j - h + 1 : 0);
                                const int yEnd = yDir ? yStart + 1 : (dim >= 2 ? j + h : 1);
                                int xStart = xDir ? (side == 0 ? i - h : i + h) : i - h;
                                int xEnd = xDir ? xStart + 1 : i + h + 1;
                                if (zDir) {
                                    xStart += 1;
                                    xEnd -= 1;
                                }
                                for (z = zStart; z < zEnd; ++z) {
                                    for (y = yStart; y < yEnd; ++y) {
                                        for (x = xStart; x < xEnd; ++x) {
                                            const double uh = value_at(u_plane, nn, gh, N, bc, x, y, z);
                                            o[h] += structure_power(fabs(u - uh), p) /
                                                (double)(nn[0] * nn[1] * nn[2]);
                                        }
                                    }
                                }
                            }
                        }
                    }
                }
            }
        }
    }
}

void orc_structure_basic(int dim, const int* n, int g, int bc, int nvar, int direction, int H,
    double p, const double* planes, double* out) {
    int nn[3], gh[3], N[3];
    long plane;
    int v, i, j, k, h;
    const int dv[3] = {direction == 0, direction == 1, direction == 2};
    structure_geometry(dim, n, g, nn, gh, N);
    plane = (long)N[0] * N[1] * N[2];
    for (v = 0; v < nvar * H; ++v) {
        out[v] = 0;
    }
    for (v = 0; v < nvar; ++v) {
        const double* u_plane = planes + v * plane;
        double* o = out + (long)v * H;
        for (k = 0; k < nn[2]; ++k) {
            for (j = 0; j < nn[1]; ++j) {
                for (i = 0; i < nn[0]; ++i) {
                    for (h = 0; h < H; ++h) {
                        const double u = u_plane[((long)(k + gh[2]) * N[1] + j + gh[1]) * N[0] + i + gh[0]];
                        const double uh = value_at(u_plane, nn, gh, N, bc, i + h * dv[0],
                            j + h * dv[1], k + h * dv[2]);
                        o[h] += pow(fabs(u - uh), p) / (double)(nn[0] * nn[1] * nn[2]);
                    }
                }
            }
        }
    }
}

/* ------------------------------------------------------- TeCNO diffusion */

/* Conserved state rotated into direction d's frame, the "rotation trick"
 * of Euler<2/3>::computeEigenVectorMatrix / computeEigenValues
 * (Euler.hpp:409-425, 506-517): 2-D d=1 m -> (m_y, -m_x); 3-D d=1
 * (m_y, -m_x, m_z), d=2 (m_z, m_y, -m_x).  Returns u (rotated), p, a. */
static void rotated_primitive(int nsd, int d, double gamma, const double* U, double* u,
    double* p, double* a) {
    double m[3] = {0, 0, 0}, dot;
    int k;
    for (k = 0; k < nsd; ++k) {
        m[k] = U[1 + k];
    }
    if (nsd == 2 && d == 1) {
        const double mx = m[0];
        m[0] = m[1];
        m[1] = -mx;
    } else if (nsd == 3 && d == 1) {
        const double mx = m[0];
        m[0] = m[1];
        m[1] = -mx;
    } else if (nsd == 3 && d == 2) {
        const double mx = m[0];
        m[0] = m[2];
        m[2] = -mx;
    }
    /* computePrimitiveVariables (Euler.hpp:290-297) */
    dot = m[0] * m[0];
    if (nsd > 1) {
        dot = dot + m[1] * m[1];
    }
    if (nsd > 2) {
        dot = dot + m[2] * m[2];
    }
    for (k = 0; k < nsd; ++k) {
        u[k] = m[k] / U[0];
    }
    *p = (gamma - 1) * (U[1 + nsd] - 0.5 * dot / U[0]);
    *a = sqrt(gamma * *p / U[0]);
}

static double udot(int nsd, const double* u) {
    double s = u[0] * u[0];
    if (nsd > 1) {
        s = s + u[1] * u[1];
    }
    if (nsd > 2) {
        s = s + u[2] * u[2];
    }
    return s;
}

/* Eigenvector matrix R[row][col] of Euler<nsd>::computeEigenVectorMatrix<d>
 * (Euler.hpp:409-466 normalised columns in 3-D, with the norm's square
 * root taken in single precision as mat.hpp:96-110 does; 506-553 in 2-D;
 * 586-623 scaled columns in 1-D). */
static void eigenvectors(int nsd, int d, double gamma, const double* U, double R[5][5]) {
    double u[3], p, a, H;
    int r, c;
    rotated_primitive(nsd, d, gamma, U, u, &p, &a);
    H = (U[1 + nsd] + p) / U[0];
    memset(R, 0, sizeof(double) * 25);
    if (nsd == 1) {
        const double rho = U[0];
        const double a1 = sqrt(rho / (2 * gamma));
        const double a2 = sqrt(rho * (gamma - 1) / gamma);
        const double a4 = a1;
        R[0][0] = a1;
        R[0][1] = a2;
        R[0][2] = a4;
        R[1][0] = a1 * (u[0] - a);
        R[1][1] = a2 * u[0];
        R[1][2] = a4 * (u[0] + a);
        R[2][0] = a1 * (H - u[0] * a);
        R[2][1] = 0.5 * a2 * udot(1, u);
        R[2][2] = a4 * (H + u[0] * a);
    } else if (nsd == 2) {
        R[0][0] = 1; R[0][1] = 1; R[0][2] = 0; R[0][3] = 1;
        R[1][0] = u[0] - a; R[1][1] = u[0]; R[1][2] = 0; R[1][3] = u[0] + a;
        R[2][0] = u[1]; R[2][1] = u[1]; R[2][2] = 1; R[2][3] = u[1];
        R[3][0] = H - u[0] * a; R[3][1] = 0.5 * udot(2, u); R[3][2] = u[1];
        R[3][3] = H + u[0] * a;
    } else {
        R[0][0] = 1; R[0][1] = 1; R[0][2] = 0; R[0][3] = 0; R[0][4] = 1;
        R[1][0] = u[0] - a; R[1][1] = u[0]; R[1][2] = 0; R[1][3] = 0; R[1][4] = u[0] + a;
        R[2][0] = u[1]; R[2][1] = u[1]; R[2][2] = 1; R[2][3] = 0; R[2][4] = u[1];
        R[3][0] = u[2]; R[3][1] = u[2]; R[3][2] = 0; R[3][3] = 1; R[3][4] = u[2];
        R[4][0] = H - u[0] * a; R[4][1] = 0.5 * udot(3, u); R[4][2] = u[1]; R[4][3] = u[2];
        R[4][4] = H + u[0] * a;
        for (c = 0; c < 5; ++c) {
            double norm = 0;
            for (r = 0; r < 5; ++r) {
                norm += R[r][c] * R[r][c];
            }
            norm = sqrtf((float)norm);
            for (r = 0; r < 5; ++r) {
                R[r][c] = R[r][c] / norm;
            }
        }
    }
}

/* Eigenvalues of the rotated flux Jacobian: u-a, u (nsd times), u+a
 * (Euler.hpp:470-498, 555-580, 646-657). */
static void eigenvalues(int nsd, int d, double gamma, const double* U, double* ev) {
    double u[3], p, a;
    int k;
    rotated_primitive(nsd, d, gamma, U, u, &p, &a);
    ev[0] = u[0] - a;
    for (k = 1; k <= nsd; ++k) {
        ev[k] = u[0];
    }
    ev[nsd + 1] = u[0] + a;
}

/* Entropy variables v(u) for E = -rho s/(gamma-1), s = log p - gamma log rho
 * (Euler.hpp:323-348). */
static void entropy_variables(int nsd, double gamma, const double* U, double* v) {
    double u[3], dot = U[1] * U[1], p, s;
    int k;
    if (nsd > 1) {
        dot = dot + U[2] * U[2];
    }
    if (nsd > 2) {
        dot = dot + U[3] * U[3];
    }
    for (k = 0; k < nsd; ++k) {
        u[k] = U[1 + k] / U[0];
    }
    p = (gamma - 1) * (U[1 + nsd] - 0.5 * dot / U[0]);
    s = log(p) - gamma * log(U[0]);
    v[0] = (gamma - s) / (gamma - 1) - (U[0] * udot(nsd, u)) / (2 * p);
    for (k = 0; k < nsd; ++k) {
        v[1 + k] = U[1 + k] / p;
    }
    v[1 + nsd] = -U[0] / p;
}

/* y = M x with the column-major accumulation of mat.hpp:47-60 (transpose:
 * M(row, col) = R[col][row]). */
static void mat_vec(int nv, double R[5][5], int transpose, const double* x, double* y) {
    int r, c;
    for (r = 0; r < nv; ++r) {
        y[r] = 0;
    }
    for (c = 0; c < nv; ++c) {
        for (r = 0; r < nv; ++r) {
            y[r] += (transpose ? R[c][r] : R[r][c]) * x[c];
        }
    }
}

int orc_diffusion_ghost_cells(int recon) {
    /* tecno::NoReconstruction: 1 (NoReconstruction.hpp:40-42); ENOCPU<order>: order */
    return recon == 0 ? 1 : recon;
}

static void load_cell(const double* planes, long plane, int nvar, long c, double* U) {
    int v;
    for (v = 0; v < nvar; ++v) {
        U[v] = planes[v * plane + c];
    }
}

/* The diffusion flux D(l, r) = 0.5 R (Lambda (left[r] - right[l])), both at
 * the mean of U[l] and U[r] (TecnoDiffusionCPU.cpp:70-88). */
static void diffusion_term(const orc_config* cfg, int d, int kind, const double* U,
    const double* rec_left, const double* rec_right, long plane, long l, long r, double* D) {
    const int nsd = cfg->dim, nv = nsd + 2;
    double Ul[5], Ur[5], avg[5], ev[5], R[5][5], diff[5], t[5], y[5];
    int k;
    load_cell(U, plane, nv, l, Ul);
    load_cell(U, plane, nv, r, Ur);
    for (k = 0; k < nv; ++k) {
        avg[k] = 0.5 * (Ur[k] + Ul[k]);
        diff[k] = rec_left[k * plane + r] - rec_right[k * plane + l];
    }
    eigenvalues(nsd, d, cfg->gamma, avg, ev);
    if (kind == 0) {
        /* RoeMatrix: diag |lambda_i| (RoeMatrix.hpp:36-45) */
        for (k = 0; k < nv; ++k) {
            t[k] = fabs(ev[k]) * diff[k];
        }
    } else {
        /* RusanovMatrix: max_i |lambda_i| (RusanovMatrix.hpp:36-54) */
        double mx = 0.0;
        for (k = 0; k < nv; ++k) {
            mx = fmax(fabs(ev[k]), mx);
        }
        for (k = 0; k < nv; ++k) {
            t[k] = mx * diff[k];
        }
    }
    eigenvectors(nsd, d, cfg->gamma, avg, R);
    mat_vec(nv, R, 0, t, y);
    for (k = 0; k < nv; ++k) {
        D[k] = 0.5 * y[k];
    }
}

void orc_diffusion_apply(const orc_config* cfg, int kind, int recon, double* state,
    const double* U, double* out) {
    int N[3];
    const int nsd = cfg->dim, nv = nsd + 2;
    const long plane = orc_plane_size(cfg);
    double* EL = state;
    double* ER = state + (long)nv * plane;
    double* OL = state + 2L * nv * plane;
    double* OR = state + 3L * nv * plane;
    double* DD = state + 4L * nv * plane;
    int d, x, y, z, k;
    padded(cfg, N);
    for (d = 0; d < nsd; ++d) {
        const long s = d == 0 ? 1 : (d == 1 ? N[0] : (long)N[0] * N[1]);
        /* pass 1: scaled entropy variables at both sides of face m-1|m for
         * m in [1, N_d - 2] along d, every transverse cell
         * (TecnoDiffusionCPU.cpp:40-58; volume_foreach.hpp:72-99) */
        for (z = 0; z < N[2]; ++z) {
            for (y = 0; y < N[1]; ++y) {
                for (x = 0; x < N[0]; ++x) {
                    const int c[3] = {x, y, z};
                    const long m = idx3(N, x, y, z);
                    double Um[5], Ul[5], avg[5], R[5][5], vm[5], vl[5], a[5], b[5];
                    if (c[d] < 1 || c[d] > N[d] - 2) {
                        continue;
                    }
                    load_cell(U, plane, nv, m, Um);
                    load_cell(U, plane, nv, m - s, Ul);
                    for (k = 0; k < nv; ++k) {
                        avg[k] = 0.5 * (Um[k] + Ul[k]);
                    }
                    eigenvectors(nsd, d, cfg->gamma, avg, R);
                    entropy_variables(nsd, cfg->gamma, Um, vm);
                    entropy_variables(nsd, cfg->gamma, Ul, vl);
                    mat_vec(nv, R, 1, vm, a);
                    mat_vec(nv, R, 1, vl, b);
                    for (k = 0; k < nv; ++k) {
                        EL[k * plane + m] = a[k];
                        ER[k * plane + m - s] = b[k];
                    }
                }
            }
        }
        /* pass 2: reconstruction of the pair (tecno/NoReconstruction.cpp:20-44
         * copies every cell; tecno/ENOCPU.cpp:35-139 for cells
         * [order-1, N_d - order + 1) along d, every transverse cell) */
        if (recon == 0) {
            memcpy(OL, EL, sizeof(double) * (size_t)nv * (size_t)plane);
            memcpy(OR, ER, sizeof(double) * (size_t)nv * (size_t)plane);
        } else {
            const int order = recon;
            int var, level;
            long i;
            for (var = 0; var < nv; ++var) {
                const double* L = EL + var * plane;
                const double* Rt = ER + var * plane;
                /* undivided differences into the operator's persistent
                 * arrays (ENOCPU.cpp:205-267): level k writes
                 * dd[k-1][j - s] for cells j with k <= c_d < N_d - k, every
                 * transverse cell; level 1 from (left, right), level k > 1
                 * from level k - 1.  Entries outside that range keep what
                 * an earlier variable, direction or call left there. */
                for (level = 1; level < order; ++level) {
                    double* out_dd = DD + (long)(level - 1) * plane;
                    const double* a = level == 1 ? L : DD + (long)(level - 2) * plane;
                    const double* b = level == 1 ? Rt : a;
                    for (i = 0; i < plane; ++i) {
                        const int c[3] = {(int)(i % N[0]), (int)((i / N[0]) % N[1]),
                            (int)(i / ((long)N[0] * N[1]))};
                        if (c[d] < level || c[d] >= N[d] - level) {
                            continue;
                        }
                        out_dd[i - s] = a[i] - b[i - s];
                    }
                }
                /* ENOCPU.cpp:84-136 for cells [order-1, N_d - order + 1) */
                for (i = 0; i < plane; ++i) {
                    const int c[3] = {(int)(i % N[0]), (int)((i / N[0]) % N[1]),
                        (int)(i / ((long)N[0] * N[1]))};
                    double w[7], uli = 0, uri = 0;
                    int shift = 0, l;
                    if (c[d] < order - 1 || c[d] >= N[d] - order + 1) {
                        continue;
                    }
                    for (level = 0; level < order - 1; ++level) {
                        /* |dd(left)| < |dd(right)| moves the stencil left */
                        if (fabs(DD[(long)level * plane + i - s]) < fabs(DD[(long)level * plane + i])) {
                            ++shift;
                        }
                    }
                    /* the stencil values are rebuilt from level-1 differences
                     * at flat offsets +l and -l-1 (ENOCPU.cpp:118-123), i.e.
                     * x-neighbours whatever the direction; kept as is */
                    w[order - 1] = L[i];
                    for (l = 0; l < order - 1; ++l) {
                        w[order + l] = w[order + l - 1] + DD[i + l];
                        w[order - l - 2] = w[order - l - 1] - DD[i - l - 1];
                    }
                    for (l = 0; l < order; ++l) {
                        uli += eno_coef(order, shift, l) * w[order - 1 - shift + l];
                        uri += eno_coef(order, shift + 1, l) * w[order - 1 - shift + l];
                    }
                    OL[var * plane + i] = uli;
                    OR[var * plane + i] = uri + (Rt[i] - L[i]);
                }
            }
        }
        /* pass 3: out[m] += D(m, m+1) - D(m-1, m) for m in [1, N_d - 2]
         * along d, every transverse cell (TecnoDiffusionCPU.cpp:62-92) */
        for (z = 0; z < N[2]; ++z) {
            for (y = 0; y < N[1]; ++y) {
                for (x = 0; x < N[0]; ++x) {
                    const int c[3] = {x, y, z};
                    const long m = idx3(N, x, y, z);
                    double Dr[5], Dl[5];
                    if (c[d] < 1 || c[d] > N[d] - 2) {
                        continue;
                    }
                    diffusion_term(cfg, d, kind, U, OL, OR, plane, m, m + s, Dr);
                    diffusion_term(cfg, d, kind, U, OL, OR, plane, m - s, m, Dl);
                    for (k = 0; k < nv; ++k) {
                        out[k * plane + m] = out[k * plane + m] + (Dr[k] - Dl[k]);
                    }
                }
            }
        }
    }
}

int orc_set_diffusion(orc_config* cfg, int kind, int recon) {
    int g;
    if ((kind != 0 && kind != 1) || (recon != 0 && (recon < 2 || recon > 4))) {
        return -1;
    }
    cfg->diffusion = kind;
    cfg->diffusion_recon = recon;
    g = orc_diffusion_ghost_cells(recon);
    if (g > cfg->g) {
        cfg->g = g;
    }
    return 0;
}

/* ------------------------------------------------------------ functionals */

/* boost::math::legendre_p(int l, double x), which Legendre.cpp:79-81 and
 * LegendrePointWise.cpp:74 call (Boost.Math special_functions/legendre.hpp,
 * not part of the reference's tree), as that library documents it under its default
 * policy: the double argument evaluated in long double (promote_double) and
 * rounded to double once at the end, a negative degree l taken as -l - 1,
 * P_0 = 1, P_1 = x and Bonnet's recurrence
 * P_{n+1} = ((2n+1) x P_n - n P_{n-1}) / (n+1), terms formed left to right.
 * |x| > 1 is Boost's domain error (an exception in the reference): here the
 * caller's flag is set and 0 returned. */
static double legendre_p(int l, double x, int* domain_error) {
    const unsigned degree = l < 0 ? (unsigned)(-l - 1) : (unsigned)l;
    const long double xl = x;
    long double p0 = 1, p1 = xl;
    unsigned m;
    if (xl < -1 || xl > 1) {
        *domain_error = 1;
        return 0;
    }
    if (degree == 0) {
        return (double)p0;
    }
    for (m = 1; m < degree; ++m) {
        const long double next = ((2 * m + 1) * xl * p1 - m * p0) / (m + 1);
        p0 = p1;
        p1 = next;
    }
    return (double)p1;
}

long orc_functional_size(int dim, const int* n, int g, int kind, int number_of_h) {
    long cells = 1, plane = 1;
    int d;
    for (d = 0; d < 3; ++d) {
        const int nd = d < dim ? n[d] : 1;
        cells *= nd;
        plane *= nd + (d < dim ? 2 * g : 0);
    }
    if (kind == ORC_FUNCTIONAL_STRUCTURE_2PT) {
        return (long)number_of_h * number_of_h;
    }
    return kind == ORC_FUNCTIONAL_IDENTITY || kind == ORC_FUNCTIONAL_LEGENDRE_POINTWISE ? cells
        : (kind == ORC_FUNCTIONAL_MOMENT ? plane : 1);
}

int orc_functional(int dim, const int* n, int g, int kind, const orc_functional_params* p,
    const double* planes, double* out, double weight) {
    int N[3], nn[3], d, i, j, k, v;
    long plane = 1;
    double len[3], sides[3], dV;
    const int nvar = dim + 2;
    long per_var;
    int domain_error = 0;
    for (d = 0; d < 3; ++d) {
        nn[d] = d < dim ? n[d] : 1;
        N[d] = nn[d] + (d < dim ? 2 * g : 0);
        plane *= N[d];
        sides[d] = p->upper[d] - p->lower[d];
        /* Grid.cpp:24-41 */
        len[d] = (p->upper[d] - p->lower[d]) / (double)nn[d];
        if (d > 0 && nn[d] == 1) {
            len[d] = 1;
        }
    }
    dV = len[0] * len[1] * len[2];
    per_var = orc_functional_size(dim, n, g, kind, p->number_of_h);
    if ((kind == ORC_FUNCTIONAL_LEGENDRE || kind == ORC_FUNCTIONAL_LEGENDRE_POINTWISE) && dim != 2) {
        return -1;
    }
    if (kind == ORC_FUNCTIONAL_BV && dim > 2) {
        return -1;
    }
    if (kind == ORC_FUNCTIONAL_BV_DIRECTION || kind == ORC_FUNCTIONAL_STRUCTURE_2PT) {
        const int dd = p->direction;
        const long s = dd == 0 ? 1 : (dd == 1 ? N[0] : (long)N[0] * N[1]);
        const int H = p->number_of_h;
        if (dd < 0 || dd >= dim) {
            return -1;
        }
        for (v = 0; v < nvar; ++v) {
            if (kind == ORC_FUNCTIONAL_BV_DIRECTION) {
                /* HostMemory::getTotalVariation(direction, p, start, end)
                 * (HostMemory.cpp:364-401): from one cell after the start
                 * along the direction */
                double bv = 0;
                for (k = 0; k < nn[2]; ++k) {
                    for (j = 0; j < nn[1]; ++j) {
                        for (i = 0; i < nn[0]; ++i) {
                            const int c[3] = {i, j, k};
                            const long idx = idx3(N, i + g, dim > 1 ? j + g : 0,
                                dim > 2 ? k + g : 0);
                            if (c[dd] == 0) {
                                continue;
                            }
                            bv += pow(fabs(planes[v * plane + idx] - planes[v * plane + idx - s]),
                                (double)p->degree);
                        }
                    }
                }
                out[v * per_var] += weight * bv;
            } else {
                /* StructureTwoPoints::computeStructure (StructureTwoPoints.cpp:48-92):
                 * per cell, for h1 then h2, accumulated in place */
                double* acc = (double*)calloc((size_t)H * H, sizeof(double));
                int h1, h2;
                const long cells = (long)nn[0] * nn[1] * nn[2];
                for (k = 0; k < nn[2]; ++k) {
                    for (j = 0; j < nn[1]; ++j) {
                        for (i = 0; i < nn[0]; ++i) {
                            const int c[3] = {i, j, k};
                            const long idx = idx3(N, i + g, dim > 1 ? j + g : 0,
                                dim > 2 ? k + g : 0);
                            const double u = planes[v * plane + idx];
                            for (h1 = 0; h1 < H; ++h1) {
                                const int a = (c[dd] + h1 < nn[dd] - 1 ? c[dd] + h1 : nn[dd] - 1) - c[dd];
                                const double u1 = planes[v * plane + idx + a * s];
                                for (h2 = 0; h2 < H; ++h2) {
                                    const int b = (c[dd] + h2 < nn[dd] - 1 ? c[dd] + h2 : nn[dd] - 1) - c[dd];
                                    const double u2 = planes[v * plane + idx + b * s];
                                    acc[h1 + H * h2] += (u1 - u) * (u1 - u) * (u2 - u) / (double)cells;
                                }
                            }
                        }
                    }
                }
                for (h1 = 0; h1 < H * H; ++h1) {
                    out[v * per_var + h1] += weight * acc[h1];
                }
                free(acc);
            }
        }
        return 0;
    }
    if (kind == ORC_FUNCTIONAL_MOMENT) {
        /* HostMemory.cpp:293-301 over every cell */
        long c;
        for (v = 0; v < nvar; ++v) {
            for (c = 0; c < plane; ++c) {
                out[v * per_var + c] += weight * pow(planes[v * plane + c], (double)p->degree);
            }
        }
        return 0;
    }
    if (kind == ORC_FUNCTIONAL_LOG_ENTROPY) {
        /* LogEntropy.cpp:30-80, midpoint loop volume_foreach.hpp:441-480 */
        double integral = 0.0;
        for (k = 0; k < nn[2]; ++k) {
            for (j = 0; j < nn[1]; ++j) {
                for (i = 0; i < nn[0]; ++i) {
                    const long idx = idx3(N, i + g, dim > 1 ? j + g : 0, dim > 2 ? k + g : 0);
                    const double rho = planes[idx];
                    const double E = planes[(nvar - 1) * plane + idx];
                    double msq = 0.0, pressure, s, ent;
                    int c;
                    for (c = 0; c < dim; ++c) {
                        const double m = planes[(1 + c) * plane + idx];
                        msq += m * m;
                    }
                    pressure = (p->gamma - 1) * (E - 1.0 / (2 * rho) * msq);
                    s = log(pressure) - p->gamma * log(rho);
                    ent = (-rho * s) / (p->gamma - 1);
                    integral += ent * dV;
                }
            }
        }
        out[(nvar - 1) * per_var] += weight * integral;
        return 0;
    }
    for (v = 0; v < nvar; ++v) {
        double integral = 0.0;
        for (k = 0; k < nn[2]; ++k) {
            for (j = 0; j < nn[1]; ++j) {
                for (i = 0; i < nn[0]; ++i) {
                    const long idx = idx3(N, i + g, dim > 1 ? j + g : 0, dim > 2 ? k + g : 0);
                    const long c = ((long)k * nn[1] + j) * nn[0] + i;
                    const double u = planes[v * plane + idx];
                    if (kind == ORC_FUNCTIONAL_IDENTITY) {
                        /* Identity.cpp:25-48 */
                        out[v * per_var + c] += weight * u;
                    } else if (kind == ORC_FUNCTIONAL_LEGENDRE_POINTWISE) {
                        /* LegendrePointWise.cpp:58-76 */
                        const double value = (u - p->min_value) / (p->max_value - p->min_value);
                        out[v * per_var + c] += legendre_p(p->degree, value, &domain_error) * weight;
                    } else if (kind == ORC_FUNCTIONAL_LEGENDRE) {
                        /* Legendre.cpp:62-90, midpoints Grid.cpp:148-171 */
                        const double x = (p->lower[0] + len[0] * i) + len[0] / 2.0;
                        const double y = (p->lower[1] + len[1] * j) + len[1] / 2.0;
                        const double xs = 2 * (x - p->lower[0]) / sides[0] - 1;
                        const double ys = 2 * (y - p->lower[1]) / sides[1] - 1;
                        const double value = (u - p->min_value) / (p->max_value - p->min_value);
                        integral += legendre_p(p->degree_k, xs, &domain_error) *
                            legendre_p(p->degree_n, ys, &domain_error) *
                            legendre_p(p->degree_m, value, &domain_error) * dV;
                    } else {
                        /* HostMemory::getTotalVariation (HostMemory.cpp:325-362):
                         * cells after the first along x and, in 2-D, y */
                        double dy = 0, dx;
                        if (i == 0 || (dim > 1 && j == 0)) {
                            continue;
                        }
                        if (dim > 1) {
                            dy = u - planes[v * plane + idx - N[0]];
                        }
                        dx = u - planes[v * plane + idx - 1];
                        integral += pow(sqrt(dy * dy + dx * dx), (double)p->degree);
                    }
                }
            }
        }
        if (kind == ORC_FUNCTIONAL_LEGENDRE || kind == ORC_FUNCTIONAL_BV) {
            out[v * per_var] += weight * integral;
        }
    }
    return domain_error ? -2 : 0;
}
