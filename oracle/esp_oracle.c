/*
 * esp_oracle.c -- FP64 C restatement of the ESP pipeline (test
 * infrastructure: the timed CPU baseline and a second oracle; never linked
 * into the product library).
 *
 * Same mathematics and stage order as oracle/esp_ref.py, following the
 * reference's stage sequence ESPForceCompute::computeForces
 * (src/ESPForceCompute.cc:96-127): cell-list neighbour list, charge
 * assignment (src/ESPForceComputeGPU.cu:206-272) with the P-segment window,
 * forward 3D FFT (src/ESPForceComputeGPU.cc:254-265), influence multiply
 * (src/ESPForceComputeGPU.cu:277-287), inverse FFT (missing in the
 * reference, src/ESPForceCompute.cc:225-232), interpolation with analytic
 * window derivatives (src/ESPForceComputeGPU.cu:292-373), the
 * EvaluatorPairPSWF pair term over the list (src/EvaluatorPairPSWF.h:274-295)
 * with the split polynomial, self and neutralising-background energies, and
 * velocity-Verlet NVE steps. Independent systems run in parallel with
 * OpenMP, one system per thread (the batched workload's natural CPU form).
 * The influence table (half spectrum) is an input, built by the numpy oracle.
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define INV_4PI 0.079577471545947673

typedef double complex cplx;

int esp_oracle_version(void) { return 2; }

/* ------------------------------------------------------------------ FFT */
/* Unnormalised DFT of n points (n 2/3/5-smooth), X_k = sum_j x_j
 * exp(sign 2 pi i j k / n), by recursive mixed-radix decimation in time.
 * tw[t] = exp(-2 pi i t / n_top); the sub-transform of length n uses every
 * (n_top / n)-th entry. */
static void fft_rec(int n, int sign, const cplx* in, int istride, cplx* out, const cplx* tw, int twstep, int ntop) {
    if (n == 1) {
        out[0] = in[0];
        return;
    }
    const int p = (n % 4 == 0) ? 4 : (n % 2 == 0) ? 2 : (n % 3 == 0) ? 3 : 5;
    const int m = n / p;
    for (int j = 0; j < p; ++j) fft_rec(m, sign, in + (size_t)j * istride, istride * p, out + (size_t)j * m, tw, twstep * p, ntop);
    cplx rootp[5];
    for (int s = 0; s < p; ++s) {
        const double a = 2.0 * M_PI * s / p;
        rootp[s] = cos(a) + (sign > 0 ? 1.0 : -1.0) * sin(a) * I;
    }
    for (int k = 0; k < m; ++k) {
        cplx t[5];
        for (int j = 0; j < p; ++j) {
            const long long e = ((long long)j * k * twstep) % ntop;
            const cplx w = sign > 0 ? conj(tw[e]) : tw[e];
            t[j] = out[(size_t)j * m + k] * w;
        }
        for (int s = 0; s < p; ++s) {
            cplx acc = 0;
            for (int j = 0; j < p; ++j) acc += t[j] * rootp[(j * s) % p];
            out[(size_t)s * m + k] = acc;
        }
    }
}

typedef struct {
    int n;
    cplx* tw;
    cplx *in, *out;
} fft_plan;

static void plan_init(fft_plan* f, int n) {
    f->n = n;
    f->tw = (cplx*)malloc(sizeof(cplx) * n);
    f->in = (cplx*)malloc(sizeof(cplx) * n);
    f->out = (cplx*)malloc(sizeof(cplx) * n);
    for (int t = 0; t < n; ++t) {
        const double a = -2.0 * M_PI * t / n;
        f->tw[t] = cos(a) + sin(a) * I;
    }
}

static void plan_free(fft_plan* f) {
    free(f->tw);
    free(f->in);
    free(f->out);
}

/* In-place transform of the lines of a 3D array a[z][y][x] along one axis. */
static void fft_axis(cplx* a, const int n[3], int axis, int sign, fft_plan* f) {
    const int nx = n[0], ny = n[1], nz = n[2];
    const size_t stride = axis == 0 ? 1 : axis == 1 ? (size_t)nx : (size_t)nx * ny;
    const int len = n[axis];
    const int o1 = axis == 0 ? ny : nx, o2 = axis == 2 ? ny : nz;
    for (int b = 0; b < o2; ++b)
        for (int c = 0; c < o1; ++c) {
            size_t base;
            if (axis == 0) base = ((size_t)b * ny + c) * nx;
            else if (axis == 1) base = (size_t)b * nx * ny + c;
            else base = (size_t)b * nx + c;
            for (int i = 0; i < len; ++i) f->in[i] = a[base + i * stride];
            fft_rec(len, sign, f->in, 1, f->out, f->tw, 1, len);
            for (int i = 0; i < len; ++i) a[base + i * stride] = f->out[i];
        }
}

/* ------------------------------------------------------------------ window */
typedef struct {
    int P, D;
    const double* wcoef; /* [P][D+1], coefficient of t^j of segment a */
} window_t;

static void weights(const window_t* w, double t, double* W, double* dW) {
    for (int a = 0; a < w->P; ++a) {
        const double* c = w->wcoef + (size_t)a * (w->D + 1);
        double v = c[w->D], d = w->D * c[w->D];
        for (int j = w->D - 1; j >= 0; --j) v = v * t + c[j];
        for (int j = w->D - 1; j >= 1; --j) d = d * t + j * c[j];
        W[a] = v;
        if (dW) dW[a] = w->D >= 1 ? d : 0.0;
    }
}

/* Mesh indices (i0 + a) mod n, a < P. */
static void stencil_index(int i0, int n, int P, int* out) {
    int v = ((i0 % n) + n) % n;
    for (int a = 0; a < P; ++a) {
        out[a] = v;
        if (++v == n) v = 0;
    }
}

/* ------------------------------------------------------------------ one system */
typedef struct {
    int N;
    double L[3];
    int n[3];
    double rcut, rlist;
    int nq;
    const double* qv; /* Q(v) = sum_j qv[j] v^j, v = 2 u - 1 */
    double lambda0, m2;
    const double* G; /* half spectrum [nz][ny][nx/2+1] */
    window_t win;
} sys_t;

static double wrap(double x, double L) {
    x -= L * floor(x / L);
    if (x >= L) x -= L;
    if (x < 0) x += L;
    return x;
}

/* Full neighbour list of all pairs with r < rlist (cell list). */
static void build_nlist(const sys_t* S, const double* pos, int** head_out, int** cnt_out, int** list_out) {
    const int N = S->N;
    int nc[3];
    for (int d = 0; d < 3; ++d) {
        nc[d] = (int)floor(S->L[d] / S->rlist);
        if (nc[d] < 1) nc[d] = 1;
    }
    const int ncell = nc[0] * nc[1] * nc[2];
    int* cell = (int*)malloc(sizeof(int) * N);
    int* cstart = (int*)calloc(ncell + 1, sizeof(int));
    int* cidx = (int*)malloc(sizeof(int) * N);
    for (int i = 0; i < N; ++i) {
        int c[3];
        for (int d = 0; d < 3; ++d) {
            c[d] = (int)(wrap(pos[3 * i + d], S->L[d]) * nc[d] / S->L[d]);
            if (c[d] >= nc[d]) c[d] = nc[d] - 1;
        }
        cell[i] = (c[2] * nc[1] + c[1]) * nc[0] + c[0];
        cstart[cell[i] + 1]++;
    }
    for (int c = 0; c < ncell; ++c) cstart[c + 1] += cstart[c];
    int* fill = (int*)calloc(ncell, sizeof(int));
    for (int i = 0; i < N; ++i) cidx[cstart[cell[i]] + fill[cell[i]]++] = i;
    int* head = (int*)malloc(sizeof(int) * N);
    int* cnt = (int*)calloc(N, sizeof(int));
    int lo[3], hi[3];
    for (int d = 0; d < 3; ++d) {
        lo[d] = nc[d] >= 3 ? -1 : 0;
        hi[d] = nc[d] >= 3 ? 1 : nc[d] - 1;
    }
    const double rl2 = S->rlist * S->rlist;
    int* list = NULL;
    size_t total = 0;
    for (int pass = 0; pass < 2; ++pass) {
        size_t off = 0;
        for (int i = 0; i < N; ++i) {
            const int ci = cell[i];
            const int cx = ci % nc[0], cy = (ci / nc[0]) % nc[1], cz = ci / (nc[0] * nc[1]);
            if (pass == 1) head[i] = (int)off;
            int k = 0;
            for (int dz = lo[2]; dz <= hi[2]; ++dz)
                for (int dy = lo[1]; dy <= hi[1]; ++dy)
                    for (int dx = lo[0]; dx <= hi[0]; ++dx) {
                        const int c = (((cz + dz + nc[2]) % nc[2]) * nc[1] + (cy + dy + nc[1]) % nc[1]) * nc[0] +
                                      (cx + dx + nc[0]) % nc[0];
                        for (int s = cstart[c]; s < cstart[c + 1]; ++s) {
                            const int j = cidx[s];
                            if (j == i) continue;
                            double r2 = 0;
                            for (int d = 0; d < 3; ++d) {
                                double x = pos[3 * i + d] - pos[3 * j + d];
                                x -= S->L[d] * round(x / S->L[d]);
                                r2 += x * x;
                            }
                            if (r2 < rl2) {
                                if (pass == 1) list[off + k] = j;
                                ++k;
                            }
                        }
                    }
            if (pass == 0) cnt[i] = k;
            off += k;
        }
        if (pass == 0) {
            total = off;
            list = (int*)malloc(sizeof(int) * (total ? total : 1));
        }
    }
    free(cell);
    free(cstart);
    free(cidx);
    free(fill);
    *head_out = head;
    *cnt_out = cnt;
    *list_out = list;
}

/* Forces F[N][3] (overwritten) and total energy of one evaluation. */
static double evaluate(const sys_t* S, const double* pos, const double* q, const int* head, const int* cnt,
                       const int* list, double* F, double* mesh_buf_re, cplx* mesh, fft_plan* fp) {
    const int N = S->N, P = S->win.P;
    const int nx = S->n[0], ny = S->n[1], nz = S->n[2], nxh = nx / 2 + 1;
    const size_t M = (size_t)nx * ny * nz;
    double W[3][16], dW[3][16];
    int i0[3];
    (void)mesh_buf_re;
    /* spread (wrapped stencil indices per axis computed once per particle) */
    int ix[16], iy[16], iz[16];
    for (size_t c = 0; c < M; ++c) mesh[c] = 0;
    for (int i = 0; i < N; ++i) {
        for (int d = 0; d < 3; ++d) {
            double g = wrap(pos[3 * i + d], S->L[d]) * (S->n[d] / S->L[d]);
            if (g >= S->n[d]) g -= S->n[d];
            i0[d] = (int)floor(g - 0.5 * P) + 1;
            weights(&S->win, i0[d] + 0.5 * P - g, W[d], NULL);
        }
        stencil_index(i0[0], nx, P, ix);
        stencil_index(i0[1], ny, P, iy);
        stencil_index(i0[2], nz, P, iz);
        for (int c = 0; c < P; ++c)
            for (int b = 0; b < P; ++b) {
                const double wzy = q[i] * W[2][c] * W[1][b];
                cplx* row = mesh + ((size_t)iz[c] * ny + iy[b]) * nx;
                for (int a = 0; a < P; ++a) row[ix[a]] += wzy * W[0][a];
            }
    }
    /* forward FFT, influence multiply, inverse FFT (unnormalised) */
    for (int axis = 0; axis < 3; ++axis) fft_axis(mesh, S->n, axis, -1, &fp[axis]);
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                double g;
                if (x < nxh) g = S->G[((size_t)z * ny + y) * nxh + x];
                else g = S->G[((size_t)((nz - z) % nz) * ny + (ny - y) % ny) * nxh + (nx - x)];
                mesh[((size_t)z * ny + y) * nx + x] *= g;
            }
    for (int axis = 0; axis < 3; ++axis) fft_axis(mesh, S->n, axis, +1, &fp[axis]);
    /* interpolation: potential and mesh force -q grad phi */
    double e_rec = 0.0;
    for (int i = 0; i < N; ++i) {
        for (int d = 0; d < 3; ++d) {
            double g = wrap(pos[3 * i + d], S->L[d]) * (S->n[d] / S->L[d]);
            if (g >= S->n[d]) g -= S->n[d];
            i0[d] = (int)floor(g - 0.5 * P) + 1;
            weights(&S->win, i0[d] + 0.5 * P - g, W[d], dW[d]);
        }
        stencil_index(i0[0], nx, P, ix);
        stencil_index(i0[1], ny, P, iy);
        stencil_index(i0[2], nz, P, iz);
        double pot = 0, gx = 0, gy = 0, gz = 0;
        for (int c = 0; c < P; ++c)
            for (int b = 0; b < P; ++b) {
                const cplx* row = mesh + ((size_t)iz[c] * ny + iy[b]) * nx;
                double sv = 0, sd = 0;
                for (int a = 0; a < P; ++a) {
                    const double ph = creal(row[ix[a]]);
                    sv += W[0][a] * ph;
                    sd += dW[0][a] * ph;
                }
                pot += W[2][c] * W[1][b] * sv;
                gx += W[2][c] * W[1][b] * sd;
                gy += W[2][c] * dW[1][b] * sv;
                gz += dW[2][c] * W[1][b] * sv;
            }
        /* dw/dr = -(n / L) dw/dt */
        F[3 * i + 0] = q[i] * gx * (nx / S->L[0]);
        F[3 * i + 1] = q[i] * gy * (ny / S->L[1]);
        F[3 * i + 2] = q[i] * gz * (nz / S->L[2]);
        e_rec += 0.5 * q[i] * pot;
    }
    /* pair term */
    const double rc = S->rcut, rc2 = rc * rc;
    const double invL[3] = {1.0 / S->L[0], 1.0 / S->L[1], 1.0 / S->L[2]};
    double e_pair = 0.0;
    for (int i = 0; i < N; ++i) {
        double fx = 0, fy = 0, fz = 0, en = 0;
        for (int k = 0; k < cnt[i]; ++k) {
            const int j = list[head[i] + k];
            double d[3], r2 = 0;
            for (int a = 0; a < 3; ++a) {
                d[a] = pos[3 * i + a] - pos[3 * j + a];
                d[a] -= S->L[a] * rint(d[a] * invL[a]);
                r2 += d[a] * d[a];
            }
            if (!(r2 < rc2) || r2 <= 0) continue;
            const double r = sqrt(r2), u = r2 / rc2, v = 2.0 * u - 1.0;
            double Q = S->qv[S->nq - 1], dQ = (S->nq - 1) * S->qv[S->nq - 1];
            for (int c = S->nq - 2; c >= 0; --c) Q = Q * v + S->qv[c];
            for (int c = S->nq - 2; c >= 1; --c) dQ = dQ * v + c * S->qv[c];
            dQ *= 2.0; /* dQ/du = 2 dQ/dv */
            const double qq = q[i] * q[j];
            en += qq * INV_4PI * (1.0 / r - Q / rc);
            const double fdr = qq * INV_4PI * (1.0 / (r2 * r) + 2.0 * dQ / (rc2 * rc));
            fx += fdr * d[0];
            fy += fdr * d[1];
            fz += fdr * d[2];
        }
        F[3 * i + 0] += fx;
        F[3 * i + 1] += fy;
        F[3 * i + 2] += fz;
        e_pair += 0.5 * en;
    }
    double qs = 0, q2 = 0;
    for (int i = 0; i < N; ++i) {
        qs += q[i];
        q2 += q[i] * q[i];
    }
    const double V = S->L[0] * S->L[1] * S->L[2];
    const double e_self = -0.5 * S->lambda0 * INV_4PI / rc * q2;
    const double e_bg = -(qs * qs) / (2.0 * V) * (rc * rc * S->m2 * 0.5);
    return e_rec + e_pair + e_self + e_bg;
}

/* Neighbour list + one evaluation + nsteps velocity-Verlet steps of one
 * system (positions and velocities updated in place, forces of the last
 * evaluation in F). Returns the energy of the last evaluation. */
static double run_system(const sys_t* S, double* pos, double* vel, const double* mass, const double* q, double* F,
                         int nsteps, double dt) {
    const int N = S->N;
    int *head, *cnt, *list;
    build_nlist(S, pos, &head, &cnt, &list);
    const size_t M = (size_t)S->n[0] * S->n[1] * S->n[2];
    cplx* mesh = (cplx*)malloc(sizeof(cplx) * M);
    fft_plan fp[3];
    for (int d = 0; d < 3; ++d) plan_init(&fp[d], S->n[d]);
    double E = evaluate(S, pos, q, head, cnt, list, F, NULL, mesh, fp);
    for (int s = 0; s < nsteps; ++s) {
        for (int i = 0; i < N; ++i)
            for (int d = 0; d < 3; ++d) {
                vel[3 * i + d] += 0.5 * dt * F[3 * i + d] / mass[i];
                pos[3 * i + d] = wrap(pos[3 * i + d] + dt * vel[3 * i + d], S->L[d]);
            }
        E = evaluate(S, pos, q, head, cnt, list, F, NULL, mesh, fp);
        for (int i = 0; i < N; ++i)
            for (int d = 0; d < 3; ++d) vel[3 * i + d] += 0.5 * dt * F[3 * i + d] / mass[i];
    }
    for (int d = 0; d < 3; ++d) plan_free(&fp[d]);
    free(mesh);
    free(head);
    free(cnt);
    free(list);
    return E;
}

/* Runs nsys independent systems (arrays concatenated; system s starts at
 * particle p_off[s], its influence table at g_off[s]) on `threads` OpenMP
 * threads, one system per thread. Window (P, D, wcoef) and split (nq, qv,
 * lambda0, m2) are shared. Returns 0. */
int esp_oracle_run_batch(int nsys, const int* N, const long long* p_off, double* pos, double* vel,
                         const double* mass, const double* q, double* F, const double* boxes, const int* meshes,
                         const long long* g_off, const double* G, int P, int D, const double* wcoef, int nq,
                         const double* qv, double lambda0, double m2, double rcut, double rlist, int nsteps, double dt,
                         double* energy, int threads) {
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 1)
#endif
    for (int s = 0; s < nsys; ++s) {
        sys_t S;
        S.N = N[s];
        for (int d = 0; d < 3; ++d) {
            S.L[d] = boxes[3 * s + d];
            S.n[d] = meshes[3 * s + d];
        }
        S.rcut = rcut;
        S.rlist = rlist;
        S.nq = nq;
        S.qv = qv;
        S.lambda0 = lambda0;
        S.m2 = m2;
        S.G = G + g_off[s];
        S.win.P = P;
        S.win.D = D;
        S.win.wcoef = wcoef;
        const long long o = p_off[s];
        energy[s] = run_system(&S, pos + 3 * o, vel + 3 * o, mass + o, q + o, F + 3 * o, nsteps, dt);
    }
    return 0;
}

int esp_oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
