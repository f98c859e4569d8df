/* CPU restatement of the DVMpp per-step hot path — the test oracle.
 *
 * TEST INFRASTRUCTURE ONLY (see dvm_oracle.h).  Parity pinned: every function
 * here is checked bit-for-bit against the reference sources compiled in
 * oracle/_ref (tests/test_oracle_vs_ref.py) and through committed golden
 * vectors generated from them (tests/golden/).
 *
 * Compiled with -ffp-contract=off: every a*b+c below is two roundings, in the
 * order the reference writes it.
 */
#define _GNU_SOURCE
#include "dvm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static const double OR_PI = 3.14159265358979323846;          /* src/BaseTypes.hpp:18 */
static const double OR_RPI2 = 1.0 / (2.0 * 3.14159265358979323846); /* src/BaseTypes.hpp:21 */

/* ---- Biot-Savart ------------------------------------------------------- */

void or_direct_self(const double* x, const double* z, const double* circ, const double* sigma,
                    size_t n, double* u, double* w) {
    /* src/VelocityKernel.cpp:37-66 */
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; ++i) {
        double ui = 0.0, wi = 0.0;
        for (size_t j = 0; j < n; ++j) {
            if ((size_t)i == j) continue;
            const double dx = x[i] - x[j];
            const double dz = z[i] - z[j];
            const double r2 = dx * dx + dz * dz;
            const double s2 = sigma[j] * sigma[j];
            const double thr = 10.0 * s2;
            const double rs = 1.0 / s2;
            double K;
            if (r2 < thr) K = (1.0 - exp(-r2 * rs)) / r2;
            else K = 1.0 / r2;
            ui -= K * dz * circ[j];
            wi += K * dx * circ[j];
        }
        u[i] = ui * OR_RPI2;
        w[i] = wi * OR_RPI2;
    }
}

void or_direct_at(const double* x, const double* z, const double* circ, const double* sigma,
                  size_t ns, const double* tx, const double* tz, size_t nt, double* u, double* w) {
    /* src/VelocityKernel.cpp:79-108 */
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)nt; ++i) {
        double ui = 0.0, wi = 0.0;
        for (size_t j = 0; j < ns; ++j) {
            const double dx = tx[i] - x[j];
            const double dz = tz[i] - z[j];
            const double r2 = dx * dx + dz * dz;
            if (r2 > 1e-15) {
                const double s2 = sigma[j] * sigma[j];
                const double thr = 10.0 * s2;
                const double rs = 1.0 / s2;
                double K;
                if (r2 < thr) K = (1.0 - exp(-r2 * rs)) / r2;
                else K = 1.0 / r2;
                ui -= K * dz * circ[j];
                wi += K * dx * circ[j];
            }
        }
        u[i] = ui * OR_RPI2;
        w[i] = wi * OR_RPI2;
    }
}

/* ---- vortex sheet ------------------------------------------------------ */

void or_sheet_geometry(const double* xp, const double* zp, int np, double* xc, double* zc,
                       double* ds, double* theta, double* enx, double* enz, double* etx,
                       double* etz) {
    /* src/VortexSheet.cpp:81-96 */
    for (int i = 0; i < np; ++i) {
        xc[i] = 0.5 * (xp[i] + xp[i + 1]);
        zc[i] = 0.5 * (zp[i] + zp[i + 1]);
        const double dx = xp[i + 1] - xp[i];
        const double dz = zp[i + 1] - zp[i];
        ds[i] = sqrt(pow(dx, 2.0) + pow(dz, 2.0));
        theta[i] = atan2(dz, dx);
        enx[i] = dz / ds[i];
        enz[i] = -dx / ds[i];
        etx[i] = -enz[i];
        etz[i] = enx[i];
    }
}

void or_influence_matrix(const double* xp, const double* zp, const double* xc, const double* zc,
                         const double* ds, const double* theta, int np, double* A) {
    /* src/VortexSheet.cpp:114-161 ; p, q are np x np, A is (np+1) x np column-major */
    const size_t m = (size_t)np + 1;
    double* p = (double*)malloc(sizeof(double) * (size_t)np * np);
    double* q = (double*)malloc(sizeof(double) * (size_t)np * np);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < np; ++i) {
        const double xci = xc[i], zci = zc[i], thi = theta[i];
        for (int j = 0; j < np; ++j) {
            double pij, qij;
            if (i == j) {
                pij = -1.0;
                qij = 1.0;
            } else {
                const double xj = xp[j], zj = zp[j], thj = theta[j], dsj = ds[j];
                const double c1 = -(xci - xj) * cos(thj) - (zci - zj) * sin(thj);
                const double c2 = pow(xci - xj, 2.0) + pow(zci - zj, 2.0);
                const double c3 = sin(thi - thj);
                const double c4 = cos(thi - thj);
                const double c5 = (xci - xj) * sin(thj) - (zci - zj) * cos(thj);
                const double c6 = log(1.0 + dsj * ((dsj + 2 * c1) / c2));
                const double c7 = atan2((c5 * dsj), (c2 + c1 * dsj));
                const double c9 = (xci - xj) * cos(thi - 2.0 * thj) - (zci - zj) * sin(thi - 2.0 * thj);
                qij = c4 + 0.5 * c9 * c6 / dsj - ((c1 * c3 + c4 * c5) * c7) / dsj;
                pij = 0.5 * c4 * c6 + c3 * c7 - qij;
            }
            p[(size_t)j * np + i] = pij;
            q[(size_t)j * np + i] = qij;
        }
    }
    for (int i = 0; i < np; ++i) {
        A[i] = -OR_RPI2 * (p[i] + q[(size_t)(np - 1) * np + i]);
        for (int j = 1; j < np; ++j)
            A[(size_t)j * m + i] = -OR_RPI2 * (p[(size_t)j * np + i] + q[(size_t)(j - 1) * np + i]);
    }
    for (int j = 0; j < np; ++j) A[(size_t)j * m + np] = ds[j];
    free(p);
    free(q);
}

void or_sheet_rhs(const double* xc, const double* zc, const double* enx, const double* enz, int np,
                  double Ux, double Uz, const double* x, const double* z, const double* circ,
                  const double* sigma, size_t n, double* b) {
    /* src/VortexSheet.cpp:171-210 */
    double tc = 0.0; /* VortexBlobs::totalcirc, src/VortexBlobs.cpp:267-270 */
    for (size_t j = 0; j < n; ++j) tc += circ[j];
    if (n == 0) {
        for (int i = 0; i < np; ++i) b[i] = Ux * enx[i] + Uz * enz[i];
        b[np] = -tc;
        return;
    }
#pragma omp parallel for schedule(static)
    for (int i = 0; i < np; ++i) {
        double ui = 0.0, wi = 0.0;
        for (size_t j = 0; j < n; ++j) {
            const double dx = xc[i] - x[j];
            const double dz = zc[i] - z[j];
            const double r2 = pow(dx, 2.0) + pow(dz, 2.0);
            const double thr = 10 * pow(sigma[j], 2.0);
            const double rs = 1.0 / pow(sigma[j], 2.0);
            double K;
            if (r2 < thr) K = (1.0 - exp(-r2 * rs)) / r2;
            else K = 1.0 / r2;
            ui -= K * dz * circ[j];
            wi += K * dx * circ[j];
        }
        ui *= OR_RPI2;
        wi *= OR_RPI2;
        b[i] = (Ux + ui) * enx[i] + (Uz + wi) * enz[i];
    }
    b[np] = -tc;
}

int or_sheet_solve(const double* A, const double* b, int np, double* gamma) {
    /* src/VortexSheet.cpp:214: arma::solve(A.t()*A, A.t()*b); the product is the
     * plain k-ordered sum and the solve is LU with partial pivoting (dgesv). */
    const size_t m = (size_t)np + 1, n = (size_t)np;
    double* N = (double*)malloc(sizeof(double) * n * n);
    double* r = (double*)malloc(sizeof(double) * n);
#pragma omp parallel for schedule(static)
    for (long jj = 0; jj < (long)n; ++jj) {
        const size_t j = (size_t)jj;
        for (size_t i = 0; i < n; ++i) {
            double acc = 0.0;
            for (size_t k = 0; k < m; ++k) acc += A[i * m + k] * A[j * m + k];
            N[j * n + i] = acc;
        }
    }
    for (size_t i = 0; i < n; ++i) {
        double acc = 0.0;
        for (size_t k = 0; k < m; ++k) acc += A[i * m + k] * b[k];
        r[i] = acc;
    }
    for (size_t k = 0; k < n; ++k) {
        size_t p = k;
        double best = fabs(N[k * n + k]);
        for (size_t i = k + 1; i < n; ++i)
            if (fabs(N[k * n + i]) > best) { best = fabs(N[k * n + i]); p = i; }
        if (best == 0.0) { free(N); free(r); return 1; }
        if (p != k) {
            for (size_t j = 0; j < n; ++j) {
                const double t = N[j * n + k]; N[j * n + k] = N[j * n + p]; N[j * n + p] = t;
            }
            const double t = r[k]; r[k] = r[p]; r[p] = t;
        }
        const double akk = N[k * n + k];
        for (size_t i = k + 1; i < n; ++i) N[k * n + i] /= akk;
#pragma omp parallel for schedule(static) if (n - k > 256)
        for (long jj = (long)k + 1; jj < (long)n; ++jj) {
            const size_t j = (size_t)jj;
            const double akj = N[j * n + k];
            if (akj == 0.0) continue;
            for (size_t i = k + 1; i < n; ++i) N[j * n + i] -= N[k * n + i] * akj;
        }
    }
    for (size_t i = 0; i < n; ++i) {
        double acc = r[i];
        for (size_t k = 0; k < i; ++k) acc -= N[k * n + i] * r[k];
        r[i] = acc;
    }
    for (size_t ii = n; ii-- > 0;) {
        double acc = r[ii];
        for (size_t k = ii + 1; k < n; ++k) acc -= N[k * n + ii] * r[k];
        r[ii] = acc / N[ii * n + ii];
    }
    memcpy(gamma, r, sizeof(double) * n);
    free(N);
    free(r);
    return 0;
}

void or_sheet_on_blobs(const double* xc, const double* zc, const double* theta, const double* ds,
                       const double* gamma, int np, const double* x, const double* z, size_t n,
                       double* uvs, double* wvs) {
    /* coefficients src/VortexSheet.cpp:225-251, accumulation :254-272 */
    const int last = np - 1;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; ++i) {
        const double xi = x[i], zi = z[i];
        double us = 0.0, ws = 0.0;
        for (int j = 0; j < np; ++j) {
            const double xj = xc[j], zj = zc[j], th = theta[j], dsj = ds[j];
            const double c1 = -(xi - xj) * cos(th) - (zi - zj) * sin(th);
            const double c2 = pow(xi - xj, 2.0) + pow(zi - zj, 2.0);
            const double c5 = (xi - xj) * sin(th) - (zi - zj) * cos(th);
            const double c6 = log(1.0 + dsj * ((dsj + 2 * c1) / c2));
            const double c7 = atan2(c5 * dsj, c2 + c1 * dsj);
            const double c8 = (xi - xj) * sin(-2.0 * th) + (zi - zj) * cos(-2.0 * th);
            const double c9 = (xi - xj) * cos(-2.0 * th) - (zi - zj) * sin(-2.0 * th);
            const double qx = -sin(th) + 0.5 * c8 * c6 / dsj + (c1 * cos(th) + c5 * sin(th)) * c7 / dsj;
            const double px = -0.5 * c6 * sin(th) - c7 * cos(th) - qx;
            const double qy = cos(th) + 0.5 * c9 * c6 / dsj + (c1 * sin(th) - c5 * cos(th)) * c7 / dsj;
            const double py = 0.5 * c6 * cos(th) - c7 * sin(th) - qy;
            const double g1 = (j == last) ? gamma[0] : gamma[j + 1];
            us += px * gamma[j] + qx * g1;
            ws += py * gamma[j] + qy * g1;
        }
        uvs[i] = us * OR_RPI2;
        wvs[i] = ws * OR_RPI2;
    }
}

/* ---- random walk, release, crossing, loads ------------------------------ */

void or_diffuse(double* x, double* z, size_t n, const double* R, double nu, double dt) {
    /* src/VortexBlobs.cpp:253-264 */
    for (size_t i = 0; i < n; ++i) {
        const double R1 = R[2 * i], R2 = R[2 * i + 1];
        const double rrw = sqrt(4.0 * nu * dt * log(1.0 / R1));
        const double th = 2.0 * OR_PI * R2;
        x[i] += rrw * cos(th);
        z[i] += rrw * sin(th);
    }
}

long or_release_counts(const double* gamma, const double* ds, int np, unsigned M, double* counts,
                       double* circ_new) {
    /* src/VortexSheet.cpp:282-297 */
    double mx = gamma[0] * ds[0];
    for (int i = 1; i < np; ++i) {
        const double pc = gamma[i] * ds[i];
        if (pc > mx) mx = pc;
    }
    double total = 0.0;
    int ok = 1;
    for (int i = 0; i < np; ++i) {
        const double pc = gamma[i] * ds[i];
        const double a = fabs(pc / mx * (double)M);
        counts[i] = floor(a) + 1.0;
        if (!(counts[i] > 1.0e-15)) ok = 0;
        circ_new[i] = pc / counts[i];
        total += counts[i];
    }
    if (!ok) return -1;
    return (long)(unsigned)total;
}

void or_release_place(const double* xp, const double* zp, const double* ds, const double* etx,
                      const double* etz, const double* enx, const double* enz, int np,
                      const double* counts, const double* circ_new, double nu, double dt,
                      double cutoff_exp, const double* R, double* x, double* z, double* circ,
                      double* sigma) {
    /* src/VortexSheet.cpp:303-331 */
    size_t c = 0;
    for (int i = 0; i < np; ++i) {
        const unsigned cnt = (unsigned)counts[i];
        for (unsigned j = 0; j < cnt; ++j) {
            const double xm = xp[i] + ds[i] * etx[i] / (counts[i] + 1);
            const double zm = zp[i] + ds[i] * etz[i] / (counts[i] + 1);
            const double rrw = fabs(sqrt(4.0 * nu * dt * log(1.0 / R[c])));
            x[c] = xm + rrw * enx[i];
            z[c] = zm + rrw * enz[i];
            circ[c] = circ_new[i];
            sigma[c] = pow(ds[i], cutoff_exp);
            ++c;
        }
    }
}

int or_inside(const double* xp, const double* zp, int np, double xc, double zc) {
    /* src/VortexSheet.cpp:450-463 */
    int cn = 0;
    for (int i = 0; i < np; ++i) {
        if (((zp[i] <= zc) && (zp[i + 1] > zc)) || ((zp[i] > zc) && (zp[i + 1] <= zc))) {
            const double vt = (zc - zp[i]) / (zp[i + 1] - zp[i]);
            if (xc < xp[i] + vt * (xp[i + 1] - xp[i])) ++cn;
        }
    }
    return cn == 1;
}

size_t or_reflect(const double* xp, const double* zp, const double* enx, const double* enz, int np,
                  double* x, double* z, size_t n) {
    /* src/VortexSheet.cpp:347-404; each blob depends only on itself */
    size_t moved = 0;
#pragma omp parallel for schedule(dynamic, 4096) reduction(+ : moved)
    for (long i = 0; i < (long)n; ++i) {
        if (!or_inside(xp, zp, np, x[i], z[i])) continue;
        const double px = x[i], pz = z[i];
        int cp = 0;
        double md = 1e10;
        for (int j = 0; j < np; ++j) {
            const double x0 = xp[j], z0 = zp[j], x1 = xp[j + 1], z1 = zp[j + 1];
            const double vx = px - x0, vz = pz - z0;
            const double dx = x1 - x0, dz = z1 - z0;
            const double len = dx * dx + dz * dz;
            double t = (vx * dx + vz * dz) / len;
            t = (t < 1.0) ? t : 1.0;  /* std::min(1.0, t) */
            t = (0.0 < t) ? t : 0.0;  /* std::max(0.0, .) */
            const double cx = x0 + t * dx, cz = z0 + t * dz;
            const double d = sqrt((px - cx) * (px - cx) + (pz - cz) * (pz - cz));
            if (d < md) { md = d; cp = j; }
        }
        const double off = 2.0 * md + 1e-6;
        x[i] = px + off * enx[cp];
        z[i] = pz + off * enz[cp];
        if (or_inside(xp, zp, np, x[i], z[i])) {
            x[i] = px + 3.0 * off * enx[cp];
            z[i] = pz + 3.0 * off * enz[cp];
        }
        ++moved;
    }
    return moved;
}

size_t or_keep_flags(const double* xp, const double* zp, int np, const double* x, const double* z,
                     size_t n, uint8_t* keep) {
    /* src/VortexSheet.cpp:413-417 */
    size_t k = 0;
#pragma omp parallel for schedule(static) reduction(+ : k)
    for (long i = 0; i < (long)n; ++i) {
        keep[i] = or_inside(xp, zp, np, x[i], z[i]) ? 0 : 1;
        k += keep[i];
    }
    return k;
}

void or_loads(const double* gamma, const double* ds, const double* enx, const double* enz, int np,
              double rho, double dt, double Ur, double* fx, double* fz) {
    /* src/VortexSheet.cpp:489-510 */
    double* P = (double*)calloc((size_t)np, sizeof(double));
    for (int i = 0; i < np - 1; ++i) P[i + 1] = P[i] + (-rho / dt * (gamma[i] * ds[i]));
    for (int i = 0; i < np - 1; ++i) P[i] = 0.5 * (P[i] + P[i + 1]);
    P[np - 1] = 0.5 * (P[np - 1] + P[0]);
    double pmax = P[0];
    for (int i = 1; i < np; ++i) if (P[i] > pmax) pmax = P[i];
    const double pref = 0.5 * rho * Ur * Ur;
    for (int i = 0; i < np; ++i) P[i] += (pref - pmax) * 1.0;
    double sx = 0.0, sz = 0.0;
    for (int i = 0; i < np; ++i) sx += P[i] * enx[i] * ds[i];
    for (int i = 0; i < np; ++i) sz += P[i] * enz[i] * ds[i];
    *fx = -sx;
    *fz = -sz;
    free(P);
}

/* ---- MT19937 + generate_canonical<double,53> ----------------------------- */

void or_mt_seed(or_mt19937* g, uint32_t seed) {
    g->mt[0] = seed;
    for (int i = 1; i < 624; ++i)
        g->mt[i] = 1812433253u * (g->mt[i - 1] ^ (g->mt[i - 1] >> 30)) + (uint32_t)i;
    g->idx = 624;
}

static uint32_t or_mt_next(or_mt19937* g) {
    if (g->idx >= 624) {
        for (int i = 0; i < 624; ++i) {
            const uint32_t y = (g->mt[i] & 0x80000000u) | (g->mt[(i + 1) % 624] & 0x7fffffffu);
            g->mt[i] = g->mt[(i + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
        }
        g->idx = 0;
    }
    uint32_t y = g->mt[g->idx++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

double or_mt_uniform(or_mt19937* g) {
    const double lo = (double)or_mt_next(g);
    const double hi = (double)or_mt_next(g);
    double r = (lo + hi * 4294967296.0) / 18446744073709551616.0;
    if (r >= 1.0) r = nextafter(1.0, 0.0);
    return r;
}

void or_mt_stream(uint32_t seed, size_t n, double* out) {
    or_mt19937 g;
    or_mt_seed(&g, seed);
    for (size_t i = 0; i < n; ++i) out[i] = or_mt_uniform(&g);
}

/* ---- whole simulation (src/DVMBase.cpp) --------------------------------- */

struct or_sim {
    or_params p;
    int np;
    double *xp, *zp, *xc, *zc, *ds, *theta, *enx, *enz, *etx, *etz, *A, *gamma, *b;
    double area, fx, fz, Ur;
    size_t n, cap;
    double *x, *z, *circ, *sigma, *u, *w, *uvs, *wvs;
    unsigned* id;
    or_mt19937 rng;
    unsigned step;
};

static void or_sim_reserve(or_sim* s, size_t need) {
    if (need <= s->cap) return;
    size_t nc = s->cap ? s->cap : 1024;
    while (nc < need) nc *= 2;
    double** arrs[] = {&s->x, &s->z, &s->circ, &s->sigma, &s->u, &s->w, &s->uvs, &s->wvs};
    for (int k = 0; k < 8; ++k) *arrs[k] = (double*)realloc(*arrs[k], nc * sizeof(double));
    s->id = (unsigned*)realloc(s->id, nc * sizeof(unsigned));
    s->cap = nc;
}

or_sim* or_sim_create(const or_params* p, const double* xp, const double* zp, int npts) {
    or_sim* s = (or_sim*)calloc(1, sizeof(or_sim));
    s->p = *p;
    s->np = npts - 1;
    const int np = s->np;
    double** arrs[] = {&s->xc, &s->zc, &s->ds, &s->theta, &s->enx, &s->enz, &s->etx, &s->etz, &s->gamma};
    for (int k = 0; k < 9; ++k) *arrs[k] = (double*)calloc((size_t)np, sizeof(double));
    s->xp = (double*)malloc(sizeof(double) * (size_t)npts);
    s->zp = (double*)malloc(sizeof(double) * (size_t)npts);
    memcpy(s->xp, xp, sizeof(double) * (size_t)npts);
    memcpy(s->zp, zp, sizeof(double) * (size_t)npts);
    s->b = (double*)calloc((size_t)np + 1, sizeof(double));
    /* src/VortexSheet.cpp:74 */
    double mx = xp[0], mn = xp[0];
    for (int i = 1; i < npts; ++i) { if (xp[i] > mx) mx = xp[i]; if (xp[i] < mn) mn = xp[i]; }
    s->area = mx - mn;
    or_sheet_geometry(xp, zp, np, s->xc, s->zc, s->ds, s->theta, s->enx, s->enz, s->etx, s->etz);
    s->A = (double*)malloc(sizeof(double) * ((size_t)np + 1) * (size_t)np);
    or_influence_matrix(xp, zp, s->xc, s->zc, s->ds, s->theta, np, s->A);
    s->Ur = sqrt(p->ux * p->ux + p->uz * p->uz); /* src/DVMBase.cpp:29 */
    or_mt_seed(&s->rng, (uint32_t)(p->seed >= 0 ? p->seed : 5489));
    or_sim_reserve(s, 1024);
    return s;
}

void or_sim_destroy(or_sim* s) {
    if (!s) return;
    double* arrs[] = {s->xp, s->zp, s->xc, s->zc, s->ds, s->theta, s->enx, s->enz, s->etx, s->etz,
                      s->A, s->gamma, s->b, s->x, s->z, s->circ, s->sigma, s->u, s->w, s->uvs, s->wvs};
    for (size_t k = 0; k < sizeof(arrs) / sizeof(arrs[0]); ++k) free(arrs[k]);
    free(s->id);
    free(s);
}

void or_sim_set_blobs(or_sim* s, size_t n, const double* x, const double* z, const double* circ,
                      const double* sigma) {
    or_sim_reserve(s, n);
    s->n = n;
    for (size_t i = 0; i < n; ++i) {
        s->x[i] = x[i]; s->z[i] = z[i]; s->circ[i] = circ[i]; s->sigma[i] = sigma[i];
        s->u[i] = s->w[i] = s->uvs[i] = s->wvs[i] = 0.0;
        s->id[i] = (unsigned)i;
    }
}

static void or_sim_velocities(or_sim* s) {
    /* DVMBase::convect stage body, src/DVMBase.cpp:172-174 / :188-193 */
    if (s->n > 0) or_direct_self(s->x, s->z, s->circ, s->sigma, s->n, s->u, s->w);
    or_sheet_rhs(s->xc, s->zc, s->enx, s->enz, s->np, s->p.ux, s->p.uz, s->x, s->z, s->circ,
                 s->sigma, s->n, s->b);
    or_sheet_solve(s->A, s->b, s->np, s->gamma);
    or_sheet_on_blobs(s->xc, s->zc, s->theta, s->ds, s->gamma, s->np, s->x, s->z, s->n, s->uvs, s->wvs);
}

static void or_sim_convect(or_sim* s) {
    /* src/DVMBase.cpp:167-209 */
    const double dt = s->p.dt, Ux = s->p.ux, Uz = s->p.uz;
    if (s->p.scheme == 0) {
        or_sim_velocities(s);
        for (size_t i = 0; i < s->n; ++i) {
            s->x[i] += (s->u[i] + s->uvs[i] + Ux) * dt;
            s->z[i] += (s->w[i] + s->wvs[i] + Uz) * dt;
        }
        return;
    }
    const double a[3] = {0, -17. / 32, -32. / 27};
    const double bb[3] = {1. / 4, 8. / 9, 3. / 4};
    double* q1 = (double*)calloc(s->n ? s->n : 1, sizeof(double));
    double* q2 = (double*)calloc(s->n ? s->n : 1, sizeof(double));
    for (int st = 0; st < 3; ++st) {
        or_sim_velocities(s);
        for (size_t i = 0; i < s->n; ++i) {
            q1[i] = a[st] * q1[i] + (s->u[i] + s->uvs[i] + Ux) * dt;
            q2[i] = a[st] * q2[i] + (s->w[i] + s->wvs[i] + Uz) * dt;
            s->x[i] += bb[st] * q1[i];
            s->z[i] += bb[st] * q2[i];
        }
    }
    free(q1);
    free(q2);
}

static int or_sim_release(or_sim* s) {
    /* src/VortexSheet.cpp:275-333 then src/VortexBlobs.cpp:211-227 */
    const int np = s->np;
    double* counts = (double*)malloc(sizeof(double) * (size_t)np);
    double* cn = (double*)malloc(sizeof(double) * (size_t)np);
    const long nrv = or_release_counts(s->gamma, s->ds, np, s->p.max_numpanelvort, counts, cn);
    if (nrv < 0) { free(counts); free(cn); return 1; }
    double* R = (double*)malloc(sizeof(double) * (size_t)(nrv ? nrv : 1));
    for (long k = 0; k < nrv; ++k) R[k] = or_mt_uniform(&s->rng);
    const size_t n0 = s->n;
    or_sim_reserve(s, n0 + (size_t)nrv);
    or_release_place(s->xp, s->zp, s->ds, s->etx, s->etz, s->enx, s->enz, np, counts, cn, s->p.nu,
                     s->p.dt, s->p.cutoff_exp, R, s->x + n0, s->z + n0, s->circ + n0, s->sigma + n0);
    for (long k = 0; k < nrv; ++k) {
        s->u[n0 + k] = s->w[n0 + k] = s->uvs[n0 + k] = s->wvs[n0 + k] = 0.0;
        s->id[n0 + k] = (unsigned)n0; /* new IDs are 0, shifted by Nold */
    }
    s->n = n0 + (size_t)nrv;
    free(R);
    free(counts);
    free(cn);
    return 0;
}

static void or_sim_delete(or_sim* s) {
    /* src/VortexSheet.cpp:407-445 */
    uint8_t* keep = (uint8_t*)malloc(s->n ? s->n : 1);
    const size_t k = or_keep_flags(s->xp, s->zp, s->np, s->x, s->z, s->n, keep);
    if (k != s->n) {
        size_t o = 0;
        for (size_t i = 0; i < s->n; ++i) {
            if (!keep[i]) continue;
            s->x[o] = s->x[i]; s->z[o] = s->z[i]; s->circ[o] = s->circ[i]; s->sigma[o] = s->sigma[i];
            s->u[o] = s->u[i]; s->w[o] = s->w[i]; s->uvs[o] = s->uvs[i]; s->wvs[o] = s->wvs[i];
            s->id[o] = (unsigned)o;
            ++o;
        }
        s->n = o;
    }
    free(keep);
}

int or_sim_phase(or_sim* s, int phase) {
    switch (phase) {
        case 0: if (s->n) or_direct_self(s->x, s->z, s->circ, s->sigma, s->n, s->u, s->w); return 0;
        case 1:
            or_sheet_rhs(s->xc, s->zc, s->enx, s->enz, s->np, s->p.ux, s->p.uz, s->x, s->z, s->circ,
                         s->sigma, s->n, s->b);
            return or_sheet_solve(s->A, s->b, s->np, s->gamma);
        case 2:
            or_sheet_on_blobs(s->xc, s->zc, s->theta, s->ds, s->gamma, s->np, s->x, s->z, s->n,
                              s->uvs, s->wvs);
            return 0;
        case 3: or_sim_convect(s); return 0;
        case 4: {
            double* R = (double*)malloc(sizeof(double) * (2 * s->n + 1));
            for (size_t k = 0; k < 2 * s->n; ++k) R[k] = or_mt_uniform(&s->rng);
            or_diffuse(s->x, s->z, s->n, R, s->p.nu, s->p.dt);
            free(R);
            return 0;
        }
        case 5: return or_sim_release(s);
        case 6:
            if (s->p.surface_cross == 0) or_sim_delete(s);
            else or_reflect(s->xp, s->zp, s->enx, s->enz, s->np, s->x, s->z, s->n);
            return 0;
        case 7:
            or_loads(s->gamma, s->ds, s->enx, s->enz, s->np, s->p.rho, s->p.dt, s->Ur, &s->fx, &s->fz);
            return 0;
        case 8: s->step++; return 0;
        case 9: or_reflect(s->xp, s->zp, s->enx, s->enz, s->np, s->x, s->z, s->n); return 0;
        case 10: or_sim_delete(s); return 0;
        default: return 2;
    }
}

int or_sim_step(or_sim* s) {
    /* src/DVMBase.cpp:86-133 (remesh disabled, merging off) */
    static const int order[] = {8, 3, 4, 5, 6, 7};
    for (int k = 0; k < 6; ++k) {
        const int rc = or_sim_phase(s, order[k]);
        if (rc) return rc;
    }
    return 0;
}

size_t or_sim_nblobs(const or_sim* s) { return s->n; }
int or_sim_npanels(const or_sim* s) { return s->np; }

void or_sim_get_blobs(const or_sim* s, double* x, double* z, double* circ, double* sigma,
                      double* u, double* w, double* uvs, double* wvs, unsigned* id) {
    const size_t n = s->n, b = n * sizeof(double);
    if (x) memcpy(x, s->x, b);
    if (z) memcpy(z, s->z, b);
    if (circ) memcpy(circ, s->circ, b);
    if (sigma) memcpy(sigma, s->sigma, b);
    if (u) memcpy(u, s->u, b);
    if (w) memcpy(w, s->w, b);
    if (uvs) memcpy(uvs, s->uvs, b);
    if (wvs) memcpy(wvs, s->wvs, b);
    if (id) memcpy(id, s->id, n * sizeof(unsigned));
}

void or_sim_get_sheet(const or_sim* s, double* gamma) {
    memcpy(gamma, s->gamma, sizeof(double) * (size_t)s->np);
}

void or_sim_get_forces(const or_sim* s, double* fx, double* fz, double* area) {
    *fx = s->fx;
    *fz = s->fz;
    if (area) *area = s->area;
}

const double* or_sim_infm(const or_sim* s) { return s->A; }


/* ---- remeshing (restated from the test formulas; see the header) ------------------ */
static double rm_w(int kernel, double r) {
    r = fabs(r);
    if (kernel == 0) {
        if (r < 1.0) return 1.0 - 2.5 * (r * r) + 1.5 * ((r * r) * r);
        if (r < 2.0) {
            const double t = 2.0 - r;
            return ((0.5 * t) * t) * (1.0 - r);
        }
        return 0.0;
    }
    if (!(r < 3.0)) return 0.0;
    if (kernel == 1) {
        double a = 3.0 - r, b = 2.0 - r, c = 1.0 - r;
        a = a > 0.0 ? ((a * a) * (a * a)) * a : 0.0;
        b = b > 0.0 ? ((b * b) * (b * b)) * b : 0.0;
        c = c > 0.0 ? ((c * c) * (c * c)) * c : 0.0;
        return ((a - 6.0 * b) + 15.0 * c) / 120.0;
    }
    return exp(-0.5 * (r * r)) * 0.398942280401432677939946;
}

size_t or_remesh(const double* x, const double* z, const double* circ, const double* sigma,
                 size_t n, double x0, double z0, double dx, double dz, int nx, int nz, int kernel,
                 double new_sigma, double threshold, double* ox, double* oz, double* oc,
                 double* os, size_t cap) {
    const int S = kernel == 0 ? 2 : 3;
    const size_t nn = (size_t)nx * (size_t)nz;
    long long* cell = (long long*)malloc(sizeof(long long) * (n ? n : 1));
    double* g = (double*)malloc(sizeof(double) * (n ? n : 1));
    size_t* cstart = (size_t*)calloc(nn + 1, sizeof(size_t));
    size_t* order = (size_t*)malloc(sizeof(size_t) * (n ? n : 1));
    double* node = (double*)malloc(sizeof(double) * nn);
    for (size_t p = 0; p < n; ++p) {
        const double xi = (x[p] - x0) / dx, ze = (z[p] - z0) / dz;
        cell[p] = -1;
        g[p] = circ[p];
        if (!(fabs(xi) < 1e9) || !(fabs(ze) < 1e9)) continue;
        const long long fx = (long long)floor(xi), fz = (long long)floor(ze);
        if (fx - (S - 1) < 0 || fx + S > nx - 1 || fz - (S - 1) < 0 || fz + S > nz - 1) continue;
        cell[p] = fz * nx + fx;
        if (kernel == 2) {
            double sx = 0.0, sz = 0.0;
            for (long long i = fx - (S - 1); i <= fx + S; ++i) sx = sx + rm_w(2, xi - (double)i);
            for (long long j = fz - (S - 1); j <= fz + S; ++j) sz = sz + rm_w(2, ze - (double)j);
            g[p] = g[p] / (sx * sz);
        }
    }
    /* stable bucketing by cell (counting sort) */
    for (size_t p = 0; p < n; ++p)
        if (cell[p] >= 0) cstart[cell[p] + 1]++;
    for (size_t c = 0; c < nn; ++c) cstart[c + 1] += cstart[c];
    {
        size_t* fill = (size_t*)malloc(sizeof(size_t) * (nn ? nn : 1));
        memcpy(fill, cstart, sizeof(size_t) * nn);
        for (size_t p = 0; p < n; ++p)
            if (cell[p] >= 0) order[fill[cell[p]]++] = p;
        free(fill);
    }
#pragma omp parallel for schedule(static)
    for (long long k = 0; k < (long long)nn; ++k) {
        const int i = (int)(k % nx), j = (int)(k / nx);
        double acc = 0.0;
        for (int b = j - S < 0 ? 0 : j - S; b <= (j + S - 1 < nz - 1 ? j + S - 1 : nz - 1); ++b)
            for (int a = i - S < 0 ? 0 : i - S; a <= (i + S - 1 < nx - 1 ? i + S - 1 : nx - 1); ++a) {
                const size_t c = (size_t)b * nx + a;
                for (size_t q = cstart[c]; q < cstart[c + 1]; ++q) {
                    const size_t p = order[q];
                    const double xi = (x[p] - x0) / dx, ze = (z[p] - z0) / dz;
                    acc = acc + (rm_w(kernel, xi - (double)i) * rm_w(kernel, ze - (double)j)) * g[p];
                }
            }
        node[k] = acc;
    }
    size_t o = 0;
    for (size_t k = 0; k < nn; ++k)
        if (fabs(node[k]) > threshold) {
            if (o < cap) {
                ox[o] = x0 + (double)(k % nx) * dx;
                oz[o] = z0 + (double)(k / nx) * dz;
                oc[o] = node[k];
                os[o] = new_sigma;
            }
            ++o;
        }
    for (size_t p = 0; p < n; ++p)
        if (cell[p] < 0) {
            if (o < cap) {
                ox[o] = x[p];
                oz[o] = z[p];
                oc[o] = circ[p];
                os[o] = sigma[p];
            }
            ++o;
        }
    free(cell);
    free(g);
    free(cstart);
    free(order);
    free(node);
    return o;
}


/* ---- vortex merging, src/VortexBlobs.cpp:110-209 ----------------------------------- */
unsigned or_merge_blobs(double* x, double* z, double* circ, double* sigma, double* u, double* w,
                        double* uvs, double* wvs, unsigned* id, size_t n, double threshold,
                        size_t* n_out) {
    *n_out = n;
    if (n < 2) return 0;
    unsigned char* merged = (unsigned char*)calloc(n, 1);
    unsigned count = 0;
    for (size_t i = 0; i < n; ++i) {
        if (merged[i]) continue;
        for (size_t j = i + 1; j < n; ++j) {
            if (merged[j]) continue;
            const double gi = circ[i], gj = circ[j];
            const double gs = gi + gj;
            if (fabs(gs) < 1e-15) continue;
            const double dx = x[i] - x[j], dz = z[i] - z[j];
            const double dist = sqrt(dx * dx + dz * dz);
            const double crit = fabs(gi * gj / gs) * dist;
            if (crit < threshold) {
                const double nx_ = (gi * x[i] + gj * x[j]) / gs;
                const double nz_ = (gi * z[i] + gj * z[j]) / gs;
                const double ns = (fabs(gi) * sigma[i] + fabs(gj) * sigma[j]) / (fabs(gi) + fabs(gj));
                x[i] = nx_;
                z[i] = nz_;
                circ[i] = gs;
                sigma[i] = ns;
                u[i] = w[i] = uvs[i] = wvs[i] = 0.0;
                merged[j] = 1;
                ++count;
            }
        }
    }
    size_t o = 0;
    if (count)
        for (size_t i = 0; i < n; ++i) {
            if (merged[i]) continue;
            x[o] = x[i]; z[o] = z[i]; circ[o] = circ[i]; sigma[o] = sigma[i];
            u[o] = u[i]; w[o] = w[i]; uvs[o] = uvs[i]; wvs[o] = wvs[i];
            id[o] = (unsigned)o;
            ++o;
        }
    else
        o = n;
    free(merged);
    *n_out = o;
    return count;
}
