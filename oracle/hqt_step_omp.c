/*
 * hqt_step_omp.c -- CPU restatement of the reference RK4 step in plain C with
 * OpenMP (TEST INFRASTRUCTURE: the timed CPU baseline and a second oracle).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU legs use it, never
 * the product path.  It restates scripts/simulation/tevol_driven_cluster.m:
 * 117-142 (the loop body) with the reference's own operators: the dense
 * spectral matrices Lx = (2*pi/L0)*fourdif(nx,1), Ly likewise (:47-48),
 * Lz = 2*chebdif(nz,1) (:49) and Lz1 = inv(Lz(1:nz-1,1:nz-1)) (:52),
 * applied along x, y and z exactly as func_Lx/func_Ly/func_Lz/func_Lzr
 * (:60-65) do, and the filter ff (src/numerics/ff.m:7-11) with the mask of
 * :27-31.  The mask keeps a Fourier mode when neither its x nor its y index
 * lies in the band, a product mx(kx)*my(ky), so ff(x) = Re(Wx x Wy^T) with
 * the circulant matrices W = F^-1 diag(m) F; for real x that is
 * Rx x Ry^T - Ix x Iy^T (R, I the real and imaginary parts of W).
 * The operator matrices come from the NumPy oracle (oracle/hqt_oracle.py,
 * pinned to the reference's known-answer tests), so this file holds the
 * step's arithmetic only.
 *
 * Every x/y derivative the right-hand side needs is computed once per stage
 * (MATLAB recomputes func_Lx(y1) in F1, F3 and F4 with identical results;
 * func_Lx(conj(y1)) = conj(func_Lx(y1)) exactly for a real matrix).
 *
 * Layout: MATLAB column-major [nx, ny, nz] (x fastest); Z1 interleaved
 * complex.  Build: see oracle/Makefile.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    int nx, ny, nz;
    double Ly_len;
    const double *Lx, *Ly, *Lz, *Lz1, *zz;  /* row-major */
    const double *Rx, *Ix, *Ry, *Iy;        /* filter matrices, row-major */
} ops_t;

/* ---- dense operators along one axis (real data, `nf` fields of size n) -- */
/* out(:, y, z) = D * in(:, y, z) */
static void along_x(const ops_t *o, const double *D, const double *in, double *out) {
    const int nx = o->nx;
    const long lines = (long)o->ny * o->nz;
#pragma omp parallel for schedule(static)
    for (long l = 0; l < lines; ++l) {
        const double *v = in + l * nx;
        double *w = out + l * nx;
        for (int i = 0; i < nx; ++i) {
            const double *d = D + (long)i * nx;
            double s = 0.0;
#pragma omp simd reduction(+ : s)
            for (int k = 0; k < nx; ++k) s += d[k] * v[k];
            w[i] = s;
        }
    }
}

/* out(x, :, z) = D * in(x, :, z) */
static void along_y(const ops_t *o, const double *D, const double *in, double *out) {
    const int nx = o->nx, ny = o->ny;
    const long plane = (long)nx * ny;
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < o->nz; ++z)
        for (int i = 0; i < ny; ++i) {
            double *w = out + z * plane + (long)i * nx;
            const double *d = D + (long)i * ny;
            for (int x = 0; x < nx; ++x) w[x] = 0.0;
            for (int k = 0; k < ny; ++k) {
                const double c = d[k];
                const double *v = in + z * plane + (long)k * nx;
#pragma omp simd
                for (int x = 0; x < nx; ++x) w[x] += c * v[x];
            }
        }
}

/* out(x, y, i) = sum_k D[i][k] in(x, y, k) for rows i < m, k < kk; rows
 * m..nz-1 of out set to zero when zero_rest (func_Lzr) */
static void along_z(const ops_t *o, const double *D, int m, int kk, int ldd, const double *in,
                    double *out) {
    const long plane = (long)o->nx * o->ny;
    const int nz = o->nz;
    const long chunk = 2048;
    const long nch = (plane + chunk - 1) / chunk;
#pragma omp parallel for schedule(static)
    for (long c = 0; c < nch; ++c) {
        const long s0 = c * chunk, s1 = s0 + chunk < plane ? s0 + chunk : plane;
        for (int i = 0; i < nz; ++i) {
            double *w = out + i * plane;
            for (long s = s0; s < s1; ++s) w[s] = 0.0;
            if (i >= m) continue;
            for (int k = 0; k < kk; ++k) {
                const double a = D[(long)i * ldd + k];
                const double *v = in + k * plane;
#pragma omp simd
                for (long s = s0; s < s1; ++s) w[s] += a * v[s];
            }
        }
    }
}

static void Lz(const ops_t *o, const double *in, double *out) {
    along_z(o, o->Lz, o->nz, o->nz, o->nz, in, out);
}
/* func_Lzr: [Lz1 * in(1:nz-1); 0] */
static void Lzr(const ops_t *o, const double *in, double *out) {
    along_z(o, o->Lz1, o->nz - 1, o->nz - 1, o->nz - 1, in, out);
}

/* ---- complex fields as separate real and imaginary planes --------------- */
typedef struct {
    double *re, *im;
} cfield;

typedef struct {
    long vol, plane;
    /* scratch */
    double *t[24];
} work_t;

static void split(const double *z, long n, double *re, double *im) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) {
        re[i] = z[2 * i];
        im[i] = z[2 * i + 1];
    }
}
static void merge(const double *re, const double *im, long n, double *z) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) {
        z[2 * i] = re[i];
        z[2 * i + 1] = im[i];
    }
}

/*
 * One RHS evaluation (tevol_driven_cluster.m:70-76) for the stage input
 * (y1 = pr + i pi, y2 = at, y3 = ax, y4 = ay); outputs k = h*F with
 * k(:,:,nz) = 0 for F1, F3, F4, and the boundary slice of h*F2 into k2b.
 * dxat, dyat: the step-constant x/y derivatives of A_t (A_t is frozen);
 * lzat: Lz(A_t), also step-constant.
 */
static void stage_rhs(const ops_t *o, work_t *W, const double *pr, const double *pi,
                      const double *at, const double *ax, const double *ay, const double *dxat,
                      const double *dyat, const double *lzat, double h, double *k1r,
                      double *k1i, double *k3, double *k4, double *k2b) {
    const long V = W->vol, P = W->plane;
    const int nz = o->nz;
    double **t = W->t;
    double *dxr = t[0], *dxi = t[1], *dyr = t[2], *dyi = t[3];
    double *lapr = t[4], *lapi = t[5], *tmp = t[6];
    double *dxax = t[7], *dyay = t[8], *dyax = t[9], *dxay = t[10];
    double *lzr = t[11], *lzi = t[12], *l2r = t[13], *l2i = t[14];
    double *g3 = t[15], *g4 = t[16], *s3 = t[17], *s4 = t[18];
    double *sr = t[19], *si = t[20];
    /* x/y derivatives, each once */
    along_x(o, o->Lx, pr, dxr);
    along_x(o, o->Lx, pi, dxi);
    along_y(o, o->Ly, pr, dyr);
    along_y(o, o->Ly, pi, dyi);
    along_x(o, o->Lx, dxr, lapr); /* Lx(Lx y1) */
    along_y(o, o->Ly, dyr, tmp);
#pragma omp parallel for schedule(static)
    for (long s = 0; s < V; ++s) lapr[s] = 0.5 * lapr[s] + 0.5 * tmp[s];
    along_x(o, o->Lx, dxi, lapi);
    along_y(o, o->Ly, dyi, tmp);
#pragma omp parallel for schedule(static)
    for (long s = 0; s < V; ++s) lapi[s] = 0.5 * lapi[s] + 0.5 * tmp[s];
    along_x(o, o->Lx, ax, dxax);
    along_y(o, o->Ly, ay, dyay);
    along_y(o, o->Ly, ax, dyax);
    along_x(o, o->Lx, ay, dxay);
    /* B-type terms: Ly(Ly y3 - Lx y4) into s3, Lx(-Ly y3 + Lx y4) into s4 */
#pragma omp parallel for schedule(static)
    for (long s = 0; s < V; ++s) tmp[s] = dyax[s] - dxay[s];
    along_y(o, o->Ly, tmp, s3);
#pragma omp parallel for schedule(static)
    for (long s = 0; s < V; ++s) tmp[s] = -dyax[s] + dxay[s];
    along_x(o, o->Lx, tmp, s4);
    /* radial derivatives of psi */
    Lz(o, pr, lzr);
    Lz(o, pi, lzi);
    Lz(o, lzr, l2r);
    Lz(o, lzi, l2i);
    /* F3, F4 inner: 0.5 Lz(d A_t + f Lz A) */
    Lz(o, ax, g3);
    Lz(o, ay, g4);
#pragma omp parallel for schedule(static)
    for (long s = 0; s < V; ++s) {
        const double z = o->zz[s / P], f = 1.0 - z * z * z;
        g3[s] = dxat[s] + f * g3[s];
        g4[s] = dyat[s] + f * g4[s];
    }
    Lz(o, g3, t[21]);
    Lz(o, g4, t[22]);
    {
        const double *lg3 = t[21], *lg4 = t[22];
#pragma omp parallel for schedule(static)
        for (long s = 0; s < V; ++s) {
            const double z = o->zz[s / P], f = 1.0 - z * z * z;
            const double a = pr[s], b = pi[s];
            const double y3 = ax[s], y4 = ay[s];
            const double mod2 = a * a + b * b;
            /* F1 argument (complex), tevol_driven_cluster.m:72-73 */
            const double lza = lzr[s], lzb = lzi[s];
            const double A_t = at[s], dA = lzat[s];
            double re = -A_t * lzb - 0.5 * b * dA + 0.5 * f * l2r[s] - 1.5 * z * z * lza -
                        0.5 * z * a - 0.5 * y3 * y3 * a - 0.5 * y4 * y4 * a + lapr[s];
            double im = A_t * lza + 0.5 * a * dA + 0.5 * f * l2i[s] - 1.5 * z * z * lzb -
                        0.5 * z * b - 0.5 * y3 * y3 * b - 0.5 * y4 * y4 * b + lapi[s];
            const double dv = dxax[s] + dyay[s];
            /* -0.5i y1 dv */
            re += 0.5 * b * dv;
            im -= 0.5 * a * dv;
            /* -i (y3 Lx y1 + y4 Ly y1) */
            const double ur = y3 * dxr[s] + y4 * dyr[s], ui = y3 * dxi[s] + y4 * dyi[s];
            re += ui;
            im -= ur;
            sr[s] = re;
            si[s] = im;
            /* F3, F4 arguments (real parts), :74-75 */
            const double imx = a * dxi[s] - b * dxr[s]; /* Im(conj(y1) Lx y1) */
            const double imy = a * dyi[s] - b * dyr[s];
            s3[s] = 0.5 * lg3[s] + 0.5 * s3[s] + imx - y3 * mod2;
            s4[s] = 0.5 * lg4[s] + 0.5 * s4[s] + imy - y4 * mod2;
        }
    }
    Lzr(o, sr, k1r);
    Lzr(o, si, k1i);
    Lzr(o, s3, k3);
    Lzr(o, s4, k4);
    /* k = h*F, k(:,:,nz) = 0 (Lzr leaves the boundary row zero already) */
#pragma omp parallel for schedule(static)
    for (long s = 0; s < V; ++s) {
        k1r[s] *= h;
        k1i[s] *= h;
        k3[s] *= h;
        k4[s] *= h;
    }
    /* F2 = (1 - z^3) Lz(Lx y3 + Ly y4), boundary row only (z = 0 there) */
    {
        const double *lzb_row = o->Lz + (long)(nz - 1) * nz;
        const double fb = 1.0 - o->zz[nz - 1] * o->zz[nz - 1] * o->zz[nz - 1];
#pragma omp parallel for schedule(static)
        for (long s = 0; s < P; ++s) {
            double acc = 0.0;
            for (int k = 0; k < nz; ++k) acc += lzb_row[k] * (dxax[k * P + s] + dyay[k * P + s]);
            k2b[s] = h * fb * acc;
        }
    }
}

static double matlab_round(double v) { return v >= 0 ? floor(v + 0.5) : -floor(-v + 0.5); }

/* filter ff of a real field in place: Rx x Ry^T - Ix x Iy^T */
static void filter_field(const ops_t *o, work_t *W, double *x) {
    const long V = W->vol;
    double *a = W->t[19], *b = W->t[20], *c = W->t[21];
    along_x(o, o->Rx, x, a);
    along_y(o, o->Ry, a, b);
    along_x(o, o->Ix, x, a);
    along_y(o, o->Iy, a, c);
#pragma omp parallel for schedule(static)
    for (long s = 0; s < V; ++s) x[s] = b[s] - c[s];
}

/*
 * Advance the state nsteps steps in place.  Z1 interleaved complex; rhoi
 * replicated along z.  windings (nsteps ints) receives the winding removed
 * at each step (0 without removal).  Returns 0, or the 1-based step at which
 * a NaN appeared (the run stops there, tevol_driven_cluster.m:182-185).
 */
int hqt_omp_run(int nx, int ny, int nz, double Ly_len, const double *Lxm, const double *Lym,
                const double *Lzm, const double *Lz1m, const double *zz, const double *Rx,
                const double *Ix, const double *Ry, const double *Iy, double *Z1, double *Z2,
                double *Z3, double *Z4, double *rhoi, int nsteps, double h, double mu,
                double vy, int remove_winding, int apply_filter, int *windings) {
    ops_t o = {nx, ny, nz, Ly_len, Lxm, Lym, Lzm, Lz1m, zz, Rx, Ix, Ry, Iy};
    work_t W;
    W.plane = (long)nx * ny;
    W.vol = W.plane * nz;
    const long V = W.vol, P = W.plane;
    for (int i = 0; i < 24; ++i) W.t[i] = (double *)malloc(sizeof(double) * V);
    double *pr = malloc(sizeof(double) * V), *pi = malloc(sizeof(double) * V);
    double *yr = malloc(sizeof(double) * V), *yi = malloc(sizeof(double) * V);
    double *y3 = malloc(sizeof(double) * V), *y4 = malloc(sizeof(double) * V);
    double *kr[4], *ki[4], *k3[4], *k4[4], *k2[4];
    for (int s = 0; s < 4; ++s) {
        kr[s] = malloc(sizeof(double) * V);
        ki[s] = malloc(sizeof(double) * V);
        k3[s] = malloc(sizeof(double) * V);
        k4[s] = malloc(sizeof(double) * V);
        k2[s] = malloc(sizeof(double) * P);
    }
    double *dxat = malloc(sizeof(double) * V), *dyat = malloc(sizeof(double) * V);
    double *lzat = malloc(sizeof(double) * V);
    double *rho = malloc(sizeof(double) * P);
    int bad = 0;
    split(Z1, V, pr, pi);
    memcpy(rho, rhoi + (long)(nz - 1) * P, sizeof(double) * P);
    const double cst[4] = {0.0, 0.5, 0.5, 1.0};
    for (int step = 0; step < nsteps && !bad; ++step) {
        /* A_t is frozen during the four stages (:120-123) */
        along_x(&o, Lxm, Z2, dxat);
        along_y(&o, Lym, Z2, dyat);
        Lz(&o, Z2, lzat);
        for (int s = 0; s < 4; ++s) {
            const double *ir = pr, *ii = pi, *i3 = Z3, *i4 = Z4;
            if (s > 0) {
                const double c = cst[s];
#pragma omp parallel for schedule(static)
                for (long q = 0; q < V; ++q) {
                    yr[q] = pr[q] + kr[s - 1][q] * c;
                    yi[q] = pi[q] + ki[s - 1][q] * c;
                    y3[q] = Z3[q] + k3[s - 1][q] * c;
                    y4[q] = Z4[q] + k4[s - 1][q] * c;
                }
                ir = yr;
                ii = yi;
                i3 = y3;
                i4 = y4;
            }
            stage_rhs(&o, &W, ir, ii, Z2, i3, i4, dxat, dyat, lzat, h, kr[s], ki[s], k3[s],
                      k4[s], k2[s]);
        }
        /* combine (:124,128) */
        const double sixth = 1.0 / 6.0;
#pragma omp parallel for schedule(static)
        for (long q = 0; q < V; ++q) {
            pr[q] = pr[q] + sixth * (kr[0][q] + 2 * kr[1][q] + 2 * kr[2][q] + kr[3][q]);
            pi[q] = pi[q] + sixth * (ki[0][q] + 2 * ki[1][q] + 2 * ki[2][q] + ki[3][q]);
            Z3[q] = Z3[q] + sixth * (k3[0][q] + 2 * k3[1][q] + 2 * k3[2][q] + k3[3][q]);
            Z4[q] = Z4[q] + sixth * (k4[0][q] + 2 * k4[1][q] + 2 * k4[2][q] + k4[3][q]);
        }
#pragma omp parallel for schedule(static)
        for (long q = 0; q < P; ++q)
            rho[q] = rho[q] - sixth * (k2[0][q] + 2 * k2[1][q] + 2 * k2[2][q] + k2[3][q]);
        /* constraint (:129-131): cons = Lz(div A) - 2 Im(conj(Z1) Lz Z1) */
        {
            double *dv = W.t[0], *t1 = W.t[1], *lr = W.t[2], *li = W.t[3], *cons = W.t[4];
            double *v = W.t[5], *lv = W.t[6];
            along_x(&o, Lxm, Z3, dv);
            along_y(&o, Lym, Z4, t1);
#pragma omp parallel for schedule(static)
            for (long q = 0; q < V; ++q) t1[q] += dv[q];
            Lz(&o, t1, cons);
            Lz(&o, pr, lr);
            Lz(&o, pi, li);
#pragma omp parallel for schedule(static)
            for (long q = 0; q < V; ++q) cons[q] -= 2.0 * (pr[q] * li[q] - pi[q] * lr[q]);
            Lzr(&o, cons, v);
#pragma omp parallel for schedule(static)
            for (long q = 0; q < V; ++q) v[q] -= rho[q % P];
            Lzr(&o, v, lv);
#pragma omp parallel for schedule(static)
            for (long q = 0; q < V; ++q) Z2[q] = lv[q] + mu;
        }
        /* boundary rows (:133) */
        for (long q = 0; q < P; ++q) {
            const long b = (long)(nz - 1) * P + q;
            pr[b] = 0.0;
            pi[b] = 0.0;
            Z3[b] = 0.0;
            Z2[b] = mu;
            Z4[b] = -vy;
        }
        /* winding removal (:136-139) */
        int w = 0;
        if (remove_winding) {
            double *Or = W.t[7], *Oi = W.t[8];
            const double *row = Lzm + (long)(nz - 1) * nz;
#pragma omp parallel for schedule(static)
            for (long q = 0; q < P; ++q) {
                double a = 0.0, b = 0.0;
                for (int k = 0; k < nz; ++k) {
                    a += row[k] * pr[k * P + q];
                    b += row[k] * pi[k * P + q];
                }
                Or[q] = a;
                Oi[q] = b;
            }
            double tot = 0.0;
            for (int j = 0; j < ny; ++j) {
                const int j1 = (j + 1) % ny;
                for (int i = 0; i < nx; ++i) {
                    const double ar = Or[(long)j1 * nx + i], ai = Oi[(long)j1 * nx + i];
                    const double br = Or[(long)j * nx + i], bi = Oi[(long)j * nx + i];
                    tot += atan2(ai * br - ar * bi, ar * br + ai * bi);
                }
            }
            w = (int)matlab_round(tot / ny / (2.0 * 3.14159265358979323846));
            if (w != 0) {
#pragma omp parallel for schedule(static)
                for (long q = 0; q < V; ++q) {
                    const long j = (q / nx) % ny;
                    const double yy = (2.0 * 3.14159265358979323846 * j / ny) * Ly_len / 2.0 /
                                      3.14159265358979323846;
                    const double ph = -2.0 * 3.14159265358979323846 * yy / Ly_len * w;
                    const double c = cos(ph), s = sin(ph);
                    const double a = pr[q], b = pi[q];
                    pr[q] = a * c - b * s;
                    pi[q] = a * s + b * c;
                }
            }
        }
        windings[step] = w;
        /* filter (:142) */
        if (apply_filter) {
            filter_field(&o, &W, pr);
            filter_field(&o, &W, pi);
            filter_field(&o, &W, Z2);
            filter_field(&o, &W, Z3);
            filter_field(&o, &W, Z4);
        }
        /* NaN guard (:182-185) */
        int nan = 0;
#pragma omp parallel for reduction(| : nan) schedule(static)
        for (long q = 0; q < V; ++q)
            nan |= isnan(pr[q]) | isnan(pi[q]) | isnan(Z2[q]) | isnan(Z3[q]) | isnan(Z4[q]);
        if (nan) bad = step + 1;
    }
    merge(pr, pi, V, Z1);
    for (int z = 0; z < nz; ++z) memcpy(rhoi + (long)z * P, rho, sizeof(double) * P);
    for (int i = 0; i < 24; ++i) free(W.t[i]);
    free(pr), free(pi), free(yr), free(yi), free(y3), free(y4);
    for (int s = 0; s < 4; ++s) free(kr[s]), free(ki[s]), free(k3[s]), free(k4[s]), free(k2[s]);
    free(dxat), free(dyat), free(lzat), free(rho);
    return bad;
}
