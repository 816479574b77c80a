/*
 * TEST INFRASTRUCTURE ONLY: the oracle's C restatement of the two particle
 * kernels of the reference lcode.py, used by tests/ and by bench.py's CPU
 * baseline. The product (liblc3d.so) neither links nor calls it.
 *
 *   oracle_move_smart  -- move_smart_kernel, lcode.py:704-793
 *   oracle_deposit     -- deposit_kernel + coarse_to_fine + weights +
 *                         deposit9, lcode.py:396-449, 576-663
 *
 * With nthreads == 1 the deposition adds the fine particles in ascending
 * index order and each particle's 9 stencil entries in the reference's order
 * (MP 0P PP M0 00 P0 MM 0M PM), i.e. the order of a serial run of the
 * reference kernel. With nthreads > 1 each thread deposits a contiguous
 * range of fine particles into a private grid and the private grids are
 * summed in thread order (deterministic for a fixed thread count).
 * Built with -ffp-contract=off so that no fused multiply-add changes the
 * rounding of the reference's expressions.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
    int i, j;
    double w[9];
} tsc_t;

/* weights(), lcode.py:396-418 */
static inline void tsc(double x, double y, int N, double h, tsc_t* t) {
    double x_h = x / h + .5, y_h = y / h + .5;
    double fx = floor(x_h), fy = floor(y_h);
    t->i = (int)fx + N / 2;
    t->j = (int)fy + N / 2;
    double xl = x_h - fx - .5, yl = y_h - fy - .5;
    double wx0 = .75 - xl * xl, wy0 = .75 - yl * yl;
    double wxP = (.5 + xl) * (.5 + xl) / 2, wyP = (.5 + yl) * (.5 + yl) / 2;
    double wxM = (.5 - xl) * (.5 - xl) / 2, wyM = (.5 - yl) * (.5 - yl) / 2;
    t->w[0] = wxM * wyP; t->w[1] = wx0 * wyP; t->w[2] = wxP * wyP;
    t->w[3] = wxM * wy0; t->w[4] = wx0 * wy0; t->w[5] = wxP * wy0;
    t->w[6] = wxM * wyM; t->w[7] = wx0 * wyM; t->w[8] = wxP * wyM;
}

static const int DI[9] = {-1, 0, +1, -1, 0, +1, -1, 0, +1};
static const int DJ[9] = {+1, +1, +1, 0, 0, 0, -1, -1, -1};

/* interp9(), lcode.py:421-430 */
static inline double interp9(const double* a, int N, const tsc_t* t) {
    double s = 0;
    for (int k = 0; k < 9; ++k) s = s + a[(t->i + DI[k]) * N + (t->j + DJ[k])] * t->w[k];
    return s;
}

/* Returns the number of particles whose stencil left the grid (skipped). */
int oracle_move_smart(int n, const double* ms, const double* qs, const double* x_init, const double* y_init,
                      const double* x_prev, const double* y_prev, const double* est_x, const double* est_y,
                      const double* px_prev, const double* py_prev, const double* pz_prev,
                      const double* Ex_a, const double* Ey_a, const double* Ez_a, const double* Bx_a,
                      const double* By_a, const double* Bz_a, int N, double h, double dxi, double rb,
                      double* out_x, double* out_y, double* out_px, double* out_py, double* out_pz,
                      int nthreads) {
    int bad = 0;
#pragma omp parallel for num_threads(nthreads) reduction(+ : bad) schedule(static)
    for (int k = 0; k < n; ++k) {
        double m = ms[k], q = qs[k];
        double opx = px_prev[k], opy = py_prev[k], opz = pz_prev[k];
        double px = opx, py = opy, pz = opz;
        double x_offt = x_prev[k], y_offt = y_prev[k];
        double xh = x_init[k] + (x_prev[k] + est_x[k]) / 2;
        double yh = y_init[k] + (y_prev[k] + est_y[k]) / 2;
        tsc_t t;
        tsc(xh, yh, N, h, &t);
        if (t.i < 1 || t.i > N - 2 || t.j < 1 || t.j > N - 2) {
            bad++;
            out_x[k] = x_offt; out_y[k] = y_offt; out_px[k] = opx; out_py[k] = opy; out_pz[k] = opz;
            continue;
        }
        double Ex = interp9(Ex_a, N, &t), Ey = interp9(Ey_a, N, &t), Ez = interp9(Ez_a, N, &t);
        double Bx = interp9(Bx_a, N, &t), By = interp9(By_a, N, &t), Bz = interp9(Bz_a, N, &t);
        double dpx = 0, dpy = 0, dpz = 0;
        for (int it = 0; it < 2; ++it) {
            double gamma_m = sqrt(m * m + pz * pz + px * px + py * py);
            double vx = px / gamma_m, vy = py / gamma_m, vz = pz / gamma_m;
            double factor_1 = q * dxi / (1 - pz / gamma_m);
            dpx = factor_1 * (Ex + vy * Bz - vz * By);
            dpy = factor_1 * (Ey - vx * Bz + vz * Bx);
            dpz = factor_1 * (Ez + vx * By - vy * Bx);
            px = opx + dpx / 2; py = opy + dpy / 2; pz = opz + dpz / 2;
        }
        double gamma_m = sqrt(m * m + pz * pz + px * px + py * py);
        x_offt += px / (gamma_m - pz) * dxi;
        y_offt += py / (gamma_m - pz) * dxi;
        px = opx + dpx; py = opy + dpy; pz = opz + dpz;
        double x = x_init[k] + x_offt, y = y_init[k] + y_offt;
        if (x > +rb) { x = +2 * rb - x; x_offt = x - x_init[k]; px = -px; }
        if (x < -rb) { x = -2 * rb - x; x_offt = x - x_init[k]; px = -px; }
        if (y > +rb) { y = +2 * rb - y; y_offt = y - y_init[k]; py = -py; }
        if (y < -rb) { y = -2 * rb - y; y_offt = y - y_init[k]; py = -py; }
        out_x[k] = x_offt; out_y[k] = y_offt; out_px[k] = px; out_py[k] = py; out_pz[k] = pz;
    }
    return bad;
}

static inline double mix(const double* c, int Nc, double A, double B, double C, double D, int pi, int ni,
                         int pj, int nj) {
    return A * c[pi * Nc + pj] + B * c[pi * Nc + nj] + C * c[ni * Nc + pj] + D * c[ni * Nc + nj];
}

static int deposit_range(long long k0, long long k1, int Nc, int Nf, int N, double h, double sf,
                         const double* cx, const double* cy, const double* cm, const double* cq,
                         const double* cpx, const double* cpy, const double* cpz, const double* ipr,
                         const double* inx, const long long* idp, const long long* idn, const double* fg,
                         double* ro, double* jx, double* jy, double* jz) {
    int bad = 0;
    for (long long fk = k0; fk < k1; ++fk) {
        int fi = (int)(fk / Nf), fj = (int)(fk % Nf);
        double A = ipr[fi] * ipr[fj], B = ipr[fi] * inx[fj], C = inx[fi] * ipr[fj], D = inx[fi] * inx[fj];
        int pi = (int)idp[fi], ni = (int)idn[fi], pj = (int)idp[fj], nj = (int)idn[fj];
        double x = fg[fi] + mix(cx, Nc, A, B, C, D, pi, ni, pj, nj);
        double y = fg[fj] + mix(cy, Nc, A, B, C, D, pi, ni, pj, nj);
        double m = sf * mix(cm, Nc, A, B, C, D, pi, ni, pj, nj);
        double q = sf * mix(cq, Nc, A, B, C, D, pi, ni, pj, nj);
        double px = sf * mix(cpx, Nc, A, B, C, D, pi, ni, pj, nj);
        double py = sf * mix(cpy, Nc, A, B, C, D, pi, ni, pj, nj);
        double pz = sf * mix(cpz, Nc, A, B, C, D, pi, ni, pj, nj);
        double gamma_m = sqrt(m * m + px * px + py * py + pz * pz);
        double dro = q / (1 - pz / gamma_m);
        double djx = px * (dro / gamma_m), djy = py * (dro / gamma_m), djz = pz * (dro / gamma_m);
        tsc_t t;
        tsc(x, y, N, h, &t);
        if (t.i < 1 || t.i > N - 2 || t.j < 1 || t.j > N - 2) {
            bad++;
            continue;
        }
        for (int k = 0; k < 9; ++k) {
            int c = (t.i + DI[k]) * N + (t.j + DJ[k]);
            ro[c] += dro * t.w[k];
            jx[c] += djx * t.w[k];
            jy[c] += djy * t.w[k];
            jz[c] += djz * t.w[k];
        }
    }
    return bad;
}

/* Outputs must be zeroed by the caller; returns the skipped-particle count. */
int oracle_deposit(int Nc, int Nf, int N, double h, double sf, const double* cx, const double* cy,
                   const double* cm, const double* cq, const double* cpx, const double* cpy, const double* cpz,
                   const double* ipr, const double* inx, const long long* idp, const long long* idn,
                   const double* fg, double* ro, double* jx, double* jy, double* jz, int nthreads) {
    const long long total = (long long)Nf * Nf;
    if (nthreads <= 1)
        return deposit_range(0, total, Nc, Nf, N, h, sf, cx, cy, cm, cq, cpx, cpy, cpz, ipr, inx, idp, idn, fg,
                             ro, jx, jy, jz);
    const size_t g = (size_t)N * N;
    double* priv = (double*)calloc((size_t)nthreads * 4 * g, sizeof(double));
    if (!priv) return -1;
    int bad = 0;
#pragma omp parallel num_threads(nthreads) reduction(+ : bad)
    {
        int t = 0, nt = 1;
#ifdef _OPENMP
        t = omp_get_thread_num();
        nt = omp_get_num_threads();
#endif
        long long k0 = total * t / nt, k1 = total * (t + 1) / nt;
        double* p = priv + (size_t)t * 4 * g;
        bad += deposit_range(k0, k1, Nc, Nf, N, h, sf, cx, cy, cm, cq, cpx, cpy, cpz, ipr, inx, idp, idn, fg,
                             p, p + g, p + 2 * g, p + 3 * g);
#pragma omp barrier
#pragma omp for schedule(static)
        for (long long c = 0; c < (long long)g; ++c) {
            for (int u = 0; u < nt; ++u) {
                const double* q = priv + (size_t)u * 4 * g;
                ro[c] += q[c];
                jx[c] += q[g + c];
                jy[c] += q[2 * g + c];
                jz[c] += q[3 * g + c];
            }
        }
    }
    free(priv);
    return bad;
}
