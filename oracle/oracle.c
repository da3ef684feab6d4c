/*
 * CPU oracle for the swept space-time hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * This file restates, in plain C, the reference's CPU arithmetic and its CPU
 * swept decomposition so that tests can check the CUDA product against it and
 * so that the benchmark can time the reference algorithm on host cores.  It is
 * never linked into the product library.
 *
 * Pinned: tests/test_oracle.py checks every function here against golden
 * frames produced by running the reference itself (the .npz files in tests/golden, made by
 * tests/golden/make_golden.py); heat/example/checker/half match bitwise and
 * Euler matches bitwise in EULER_SQUARE_POW mode.
 *
 * Arithmetic follows the numpy CPU plugins operation by operation (no FMA
 * contraction: build with -ffp-contract=off):
 *   heat      pysweep/equations/heat.py:21-31 (step), :48-64 (forwardEuler,
 *             rungeKuttaTwo, centralDifference), courant = alpha*dt/dx/dx
 *             (heat.py:37)
 *   euler     pysweep/equations/euler.py:131-313
 *   example   pysweep/equations/example.py:13-26
 *   checker   pysweep/equations/checker.py:13-33
 *   half      pysweep/equations/half.py:15-19, :35-39
 * Swept decomposition follows pysweep/core/solver.py:113-128,158-176,
 * pysweep/core/functions.py:12-123, pysweep/core/block.py:45-62,106-164,
 * pysweep/core/geometry.py:26-36 and pysweep/core/io.py:134-144.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

enum { EQ_HEAT = 0, EQ_EULER = 1, EQ_EXAMPLE = 2, EQ_CHECKER = 3, EQ_HALF = 4 };
enum { EULER_SQUARE_POW = 0, EULER_SQUARE_MUL = 1 };

/* Neighbour offsets: xo[k] / yo[k] is the element offset of the point at
 * distance k-2 in x (rows) / y (columns) from the centre. */
typedef struct {
    long xo[5];
    long yo[5];
    long vs; /* variable stride */
} nbr_t;

/* ----------------------------------------------------------------- heat -- */
/* heat.py:60-64: courant*(u[x+1]-2*u[x]+u[x-1]) + courant*(u[y+1]-2*u+u[y-1]) */
static inline double heat_cd(const double *u, const nbr_t *n, double courant)
{
    double c = u[0];
    double dx2 = courant * ((u[n->xo[3]] - 2.0 * c) + u[n->xo[1]]);
    double dy2 = courant * ((u[n->yo[3]] - 2.0 * c) + u[n->yo[1]]);
    return dx2 + dy2;
}

static void heat_cell(const double *cur, const double *prev, double *out, const nbr_t *n,
                      const double *p, int gts)
{
    double courant = p[0];
    if (p[1] != 0.0) { /* forwardEuler: heat.py:48-51 */
        out[0] = heat_cd(cur, n, courant) + cur[0];
    } else { /* rungeKuttaTwo: heat.py:53-57 */
        int full = (gts % 2 == 0);
        double coeff = full ? 1.0 : 0.5;
        const double *base = full ? prev : cur;
        out[0] = coeff * heat_cd(cur, n, courant) + base[0];
    }
}

/* ----------------------------------------------------------------- half -- */
static inline double half_cd(const double *u, const nbr_t *n)
{
    double c = u[0];
    double a = ((u[n->xo[3]] - 2.0 * c) + u[n->xo[1]]) / 100.0;
    double b = ((u[n->yo[3]] - 2.0 * c) + u[n->yo[1]]) / 100.0;
    return a + b;
}

static void half_cell(const double *cur, const double *prev, double *out, const nbr_t *n,
                      const double *p, int gts)
{
    (void)p;
    int full = (gts % 2 == 0);
    double coeff = full ? 1.0 : 0.5;
    const double *base = full ? prev : cur;
    out[0] = base[0] + coeff * half_cd(cur, n);
}

/* -------------------------------------------------------------- example -- */
static void example_cell(const double *cur, const double *prev, double *out, const nbr_t *n,
                         const double *p, int gts)
{
    for (int v = 0; v < (int)p[1]; ++v) {
        long o = v * n->vs;
        if (p[0] != 0.0) {
            out[o] = cur[o] + 1.0;
        } else {
            int full = (gts % 2 == 0);
            out[o] = (full ? prev[o] : cur[o]) + (full ? 2.0 : 1.0);
        }
    }
}

/* -------------------------------------------------------------- checker -- */
static void checker_cell(const double *cur, const double *prev, double *out, const nbr_t *n,
                         const double *p, int gts)
{
    (void)prev;
    (void)gts;
    for (int v = 0; v < (int)p[1]; ++v) {
        long o = v * n->vs;
        double s = cur[o + n->xo[3]];
        s += cur[o + n->xo[1]];
        s += cur[o + n->yo[3]];
        s += cur[o + n->yo[1]];
        out[o] = s / 4.0;
    }
}

/* ---------------------------------------------------------------- euler -- */
typedef struct {
    double gamma, gm1;
    int sqmode;
} euler_c;

static inline double sq(const euler_c *e, double x)
{
    /* numpy evaluates float64**2 through libm pow(); pow(x,2) is not always
     * the correctly rounded x*x, so the oracle can follow either. */
    /* The exponent is read through a volatile so that the compiler cannot
     * rewrite pow(x, 2.0) as x*x. */
    static volatile double two = 2.0;
    return e->sqmode == EULER_SQUARE_POW ? pow(x, two) : x * x;
}

/* euler.py:284-293 */
static inline double e_pressure(const euler_c *e, const double q[4])
{
    return e->gm1 * (q[3] - (q[1] * q[1] + q[2] * q[2]) / (2.0 * q[0]));
}

/* euler.py:250-256 */
static inline void e_limiter(const double s1[4], const double s2[4], double num, double den,
                             double out[4])
{
    double pr = num / den;
    if (isnan(pr) || isinf(pr) || pr > 1e6 || pr < 0.0)
        pr = 0.0;
    double h = (1.0 < pr ? 1.0 : pr) / 2.0;
    for (int v = 0; v < 4; ++v)
        out[v] = s1[v] + h * (s2[v] - s1[v]);
}

/* euler.py:181-197 (dir=1) and :225-241 (dir=2) */
static inline void e_flux(const euler_c *e, const double L[4], const double R[4], int dir,
                          double f[4])
{
    double pl = e_pressure(e, L), pr = e_pressure(e, R);
    if (dir == 1) {
        f[0] = L[1] + R[1];
        f[1] = ((sq(e, L[1]) / L[0] + pl) + sq(e, R[1]) / R[0]) + pr;
        f[2] = (L[1] * L[2]) / L[0] + (R[1] * R[2]) / R[0];
        f[3] = ((L[3] + pl) * L[1]) / L[0] + ((R[3] + pr) * R[1]) / R[0];
    } else {
        f[0] = L[2] + R[2];
        f[1] = (L[1] * L[2]) / L[0] + (R[1] * R[2]) / R[0];
        f[2] = ((sq(e, L[2]) / L[0] + pl) + sq(e, R[2]) / R[0]) + pr;
        f[3] = ((L[3] + pl) * L[2]) / L[0] + ((R[3] + pr) * R[2]) / R[0];
    }
}

/* euler.py:258-282 */
static inline void e_spectral(const euler_c *e, const double L[4], const double R[4], int dir,
                              double s[4])
{
    double rl = sqrt(L[0]), rr = sqrt(R[0]);
    double tl[4], tr[4], sp[4], spv[4];
    for (int v = 0; v < 4; ++v) {
        tl[v] = L[v] / L[0];
        tr[v] = R[v] / R[0];
    }
    double denom = 1.0 / (rl + rr);
    sp[0] = rl * rr;
    for (int v = 1; v < 4; ++v)
        sp[v] = (rl * tl[v] + rr * tr[v]) * denom;
    spv[0] = sp[0];
    spv[1] = sp[0] * sp[1];
    spv[2] = sp[0] * sp[2];
    spv[3] = sp[0] * sp[3];
    double p = e_pressure(e, spv);
    double rad = sqrt(e->gamma * p / sp[0]) + fabs(sp[dir]);
    if (isnan(rad))
        rad = 0.0;
    for (int v = 0; v < 4; ++v)
        s[v] = rad * (L[v] - R[v]);
}

static inline void e_load(const double *u, long off, long vs, double q[4])
{
    for (int v = 0; v < 4; ++v)
        q[v] = u[off + v * vs];
}

/* euler.py:158-179 (dir=1, offsets xo) / :202-223 (dir=2, offsets yo) */
static void e_dflux(const euler_c *e, const double *u, const long *o, long vs, int dir,
                    double out[4])
{
    double q[5][4], P[5];
    for (int k = 0; k < 5; ++k) {
        e_load(u, o[k], vs, q[k]);
        P[k] = e_pressure(e, q[k]);
    }
    /* k: 0=ww 1=w 2=c 3=e 4=ee */
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    double L[4], R[4], f[4], s[4];
    e_limiter(q[1], q[2], P[2] - P[1], P[1] - P[0], L);
    e_limiter(q[2], q[1], P[2] - P[1], P[3] - P[2], R);
    e_flux(e, L, R, dir, f);
    e_spectral(e, L, R, dir, s);
    for (int v = 0; v < 4; ++v) {
        acc[v] += f[v];
        acc[v] += s[v];
    }
    e_limiter(q[2], q[3], P[3] - P[2], P[2] - P[1], L);
    e_limiter(q[3], q[2], P[3] - P[2], P[4] - P[3], R);
    e_flux(e, L, R, dir, f);
    e_spectral(e, L, R, dir, s);
    for (int v = 0; v < 4; ++v) {
        acc[v] -= f[v];
        acc[v] -= s[v];
    }
    for (int v = 0; v < 4; ++v)
        out[v] = acc[v] * 0.5;
}

/* euler.py:131-151.  p = {dtdx, dtdy, gamma, gm1, sqmode} */
static void euler_cell(const double *cur, const double *prev, double *out, const nbr_t *n,
                       const double *p, int gts)
{
    euler_c e = {p[2], p[3], (int)p[4]};
    double fx[4], fy[4];
    e_dflux(&e, cur, n->xo, n->vs, 1, fx);
    e_dflux(&e, cur, n->yo, n->vs, 2, fy);
    double dtdx = p[0], dtdy = p[1];
    if (gts % 2 == 0) {
        for (int v = 0; v < 4; ++v)
            out[v * n->vs] = prev[v * n->vs] + (fx[v] * dtdx + fy[v] * dtdy);
    } else {
        for (int v = 0; v < 4; ++v)
            out[v * n->vs] = cur[v * n->vs] + 0.5 * (fx[v] * dtdx + fy[v] * dtdy);
    }
}

typedef void (*cell_fn)(const double *, const double *, double *, const nbr_t *,
                        const double *, int);

static cell_fn pick(int eq)
{
    switch (eq) {
    case EQ_HEAT: return heat_cell;
    case EQ_EULER: return euler_cell;
    case EQ_EXAMPLE: return example_cell;
    case EQ_CHECKER: return checker_cell;
    case EQ_HALF: return half_cell;
    default: return NULL;
    }
}

/* ------------------------------------------------- standard (periodic) -- */
/*
 * Advance a periodic field level by level.  levels[0..its-1] hold the base
 * levels (oldest first); the result after each computed level L (global time
 * step gts = gts0 + L - 1, the reference starts at 1) is the new current
 * level.  A frame is stored every time gts % its == 0, which is when the
 * reference's writers store one (io.py:137, io.py:189).
 *
 * u: [nv][nx][ny] current level (in/out), up: previous level (in/out).
 * frames: nullable, [max_frames][nv][nx][ny]; returns number of frames.
 */
long oracle_standard(int eq, const double *p, int nv, int nx, int ny, int its, double *u,
                     double *up, long nlevels, int gts0, double *frames, long max_frames,
                     int nthreads)
{
    cell_fn f = pick(eq);
    if (!f)
        return -1;
    long N = (long)nv * nx * ny;
    double *nxt = (double *)malloc(sizeof(double) * N);
    if (!nxt)
        return -2;
    long nframes = 0;
    (void)nthreads;
    for (long L = 0; L < nlevels; ++L) {
        int gts = gts0 + (int)L;
#pragma omp parallel for num_threads(nthreads) schedule(static)
        for (int x = 0; x < nx; ++x) {
            nbr_t nb;
            nb.vs = (long)nx * ny;
            for (int k = 0; k < 5; ++k)
                nb.xo[k] = (long)(((x + k - 2 + 2 * nx) % nx) - x) * ny;
            for (int y = 0; y < ny; ++y) {
                for (int k = 0; k < 5; ++k)
                    nb.yo[k] = ((y + k - 2 + 2 * ny) % ny) - y;
                long c = (long)x * ny + y;
                f(u + c, up + c, nxt + c, &nb, p, gts);
            }
        }
        memcpy(up, u, sizeof(double) * N);
        memcpy(u, nxt, sizeof(double) * N);
        if (frames && gts % its == 0 && nframes < max_frames)
            memcpy(frames + nframes++ * N, u, sizeof(double) * N);
    }
    free(nxt);
    (void)its;
    return nframes;
}

/* ---------------------------------------------------- swept (CPU path) -- */
/*
 * Restatement of the reference's CPU swept decomposition on one node with
 * share = 0.  The window W holds T = 2*MPSS+ITS time levels of the whole
 * domain ([T][nv][nx][ny]).  Each phase copies one bs x bs block (all T
 * levels) into a block-local array, applies the phase's index sets level by
 * level (block.py:123-164), and copies the block back
 * (geometry.py:26-36).  Blocks of one phase are independent, so they are
 * processed in parallel, as the reference spreads them over MPI ranks.
 */
typedef struct {
    int lo_x, hi_x, lo_y, hi_y;
} rect_t;

typedef struct {
    int bs, ops, its, mpss, T, nv, nx, ny;
    int eq;
    const double *p;
    double *W;
    int nthreads;
} swept_t;

/* Index set of phase `ph`, level k (block-local rectangle). */
enum { PH_UP = 0, PH_DOWN = 1, PH_XB = 2, PH_YB = 3, PH_OCT = 4 };

static rect_t phase_rect(const swept_t *s, int ph, int k)
{
    int bs = s->bs, ops = s->ops, h = bs / 2, M = s->mpss;
    rect_t r;
    switch (ph) {
    case PH_UP: /* createUpPyramidSets */
        r.lo_x = r.lo_y = ops * (k + 1);
        r.hi_x = r.hi_y = bs - ops * (k + 1);
        break;
    case PH_DOWN: /* createDownPyramidSets */
        r.lo_x = r.lo_y = h - ops * (k + 1);
        r.hi_x = r.hi_y = h + ops * (k + 1);
        break;
    case PH_YB: /* createBridgeSets, first result */
        r.lo_x = ops * (k + 1);
        r.hi_x = bs - ops * (k + 1);
        r.lo_y = h - ops * (k + 1);
        r.hi_y = h + ops * (k + 1);
        break;
    case PH_XB: /* createBridgeSets, reversed */
    {
        int i = M - 1 - k;
        r.lo_x = ops * (i + 1);
        r.hi_x = bs - ops * (i + 1);
        r.lo_y = h - ops * (i + 1);
        r.hi_y = h + ops * (i + 1);
        /* product(arange(xdl,xul), arange(ydl,yul)) of set i: rows are the
         * first factor. */
        break;
    }
    default: /* PH_OCT: down sets then up sets */
        if (k < M)
            return phase_rect(s, PH_DOWN, k);
        return phase_rect(s, PH_UP, k - M);
    }
    return r;
}

static int phase_nsets(const swept_t *s, int ph)
{
    return ph == PH_OCT ? 2 * s->mpss : s->mpss;
}

/* One block: rows [bx, bx+bs), columns [by, by+bs) of W, columns wrap. */
static void run_block(const swept_t *s, int ph, int start, int gts, int bx, int by, double *loc)
{
    int bs = s->bs, T = s->T, nv = s->nv, ny = s->ny;
    long wl = (long)nv * s->nx * ny, wv = (long)s->nx * ny;
    long ll = (long)nv * bs * bs, lv = (long)bs * bs;
    for (int t = 0; t < T; ++t)
        for (int v = 0; v < nv; ++v)
            for (int i = 0; i < bs; ++i) {
                const double *src = s->W + t * wl + v * wv + (long)(bx + i) * ny;
                double *dst = loc + t * ll + v * lv + (long)i * bs;
                for (int j = 0; j < bs; ++j)
                    dst[j] = src[(by + j) % ny];
            }
    cell_fn f = pick(s->eq);
    nbr_t nb;
    nb.vs = lv;
    for (int k = 0; k < 5; ++k) {
        nb.xo[k] = (long)(k - 2) * bs;
        nb.yo[k] = k - 2;
    }
    int ns = phase_nsets(s, ph);
    for (int k = 0; k < ns; ++k) {
        rect_t r = phase_rect(s, ph, k);
        int ts = start + k, ct = gts + k;
        for (int x = r.lo_x; x < r.hi_x; ++x)
            for (int y = r.lo_y; y < r.hi_y; ++y) {
                long c = (long)x * bs + y;
                f(loc + ts * ll + c, loc + (ts - 1) * ll + c, loc + (ts + 1) * ll + c, &nb, s->p,
                  ct);
            }
    }
    for (int t = 0; t < T; ++t)
        for (int v = 0; v < nv; ++v)
            for (int i = 0; i < bs; ++i) {
                double *dst = s->W + t * wl + v * wv + (long)(bx + i) * ny;
                const double *src = loc + t * ll + v * lv + (long)i * bs;
                for (int j = 0; j < bs; ++j)
                    dst[(by + j) % ny] = src[j];
            }
}

static void run_phase(const swept_t *s, int ph, int start, int gts, int edge)
{
    int nbx = s->nx / s->bs, nby = s->ny / s->bs, nb = nbx * nby;
    int shift = edge ? s->bs / 2 : 0;
#pragma omp parallel num_threads(s->nthreads)
    {
        double *loc = (double *)malloc(sizeof(double) * s->T * s->nv * s->bs * s->bs);
#pragma omp for schedule(dynamic, 1)
        for (int b = 0; b < nb; ++b) {
            int j = b / nbx, i = b % nbx; /* block.py: columns outer, rows inner */
            run_block(s, ph, start, gts, i * s->bs, j * s->bs + shift, loc);
        }
        free(loc);
    }
}

/* Roll all window rows by +d (new[r] = old[r-d]) (functions.py:90-123). */
static void roll_rows(const swept_t *s, int d, double *tmp)
{
    long rowsz = s->ny;
    long plane = (long)s->nx * s->ny;
    int nx = s->nx;
    for (long tv = 0; tv < (long)s->T * s->nv; ++tv) {
        double *P = s->W + tv * plane;
        memcpy(tmp, P, sizeof(double) * plane);
        for (int r = 0; r < nx; ++r)
            memcpy(P + r * rowsz, tmp + (long)(((r - d) % nx + nx) % nx) * rowsz,
                   sizeof(double) * rowsz);
    }
}

/* Slide the window down by MPSS levels, storing completed frames (io.py:134-144). */
static long window_write(const swept_t *s, int gts, int sub, double *frames, long nframes,
                         long max_frames)
{
    long plane = (long)s->nv * s->nx * s->ny;
    for (int i = (gts + sub) % s->its + s->its; i < s->mpss + s->its; i += s->its)
        if (frames && nframes < max_frames)
            memcpy(frames + nframes++ * plane, s->W + i * plane, sizeof(double) * plane);
        else
            nframes++;
    int nte = s->T - s->mpss;
    memmove(s->W, s->W + (long)s->mpss * plane, sizeof(double) * plane * nte);
    return nframes;
}

/*
 * Full reference CPU swept run (solver.py:158-176).  ic: [nv][nx][ny];
 * max_gss: maxGlobalSweptStep (number of UpPrism calls).  frames (nullable):
 * receives frame 0 = ic and every completed frame the reference would write.
 * final_out (nullable): window level (ITS-1) at the end, i.e. the last
 * completed level.  Returns the number of frames.
 */
long oracle_swept(int eq, const double *p, int nv, int nx, int ny, int its, int ops, int bs,
                  int max_gss, const double *ic, double *frames, long max_frames,
                  double *final_out, int nthreads)
{
    swept_t s;
    s.bs = bs;
    s.ops = ops;
    s.its = its;
    s.mpss = bs / (2 * ops) - 1;
    s.T = 2 * s.mpss + its;
    s.nv = nv;
    s.nx = nx;
    s.ny = ny;
    s.eq = eq;
    s.p = p;
    s.nthreads = nthreads > 0 ? nthreads : 1;
    if (s.mpss < 1 || nx % bs || ny % bs || !pick(eq))
        return -1;
    long plane = (long)nv * nx * ny;
    s.W = (double *)calloc((size_t)s.T * plane, sizeof(double));
    double *tmp = (double *)malloc(sizeof(double) * nx * ny);
    if (!s.W || !tmp)
        return -2;
    for (int i = 0; i < its; ++i)
        memcpy(s.W + i * plane, ic, sizeof(double) * plane);
    long nframes = 0;
    if (frames && max_frames > 0)
        memcpy(frames, ic, sizeof(double) * plane);
    nframes = 1;
    int sub = (s.mpss % 2 != 0 && its % 2 == 0) ? 1 : 0;
    int split = bs / 2;
    int gts = 1;
    int start = its - 1;
    /* FirstPrism: Up on edge blocks, Y-bridge on blocks */
    run_phase(&s, PH_UP, start, gts, 1);
    run_phase(&s, PH_YB, start, gts, 0);
    int yb_start = start + s.mpss;
    roll_rows(&s, split, tmp); /* firstForward */
    int backward = 1;
    for (int it = 0; it < max_gss; ++it) {
        /* UpPrism */
        run_phase(&s, PH_XB, start, gts, 0);
        run_phase(&s, PH_OCT, start, gts, 1);
        gts += s.mpss;
        run_phase(&s, PH_YB, yb_start, gts, 0);
        if (backward) { /* sendBackward: shift then write */
            roll_rows(&s, -split, tmp);
            nframes = window_write(&s, gts, sub, frames, nframes, max_frames);
        } else { /* sendForward: write then shift */
            nframes = window_write(&s, gts, sub, frames, nframes, max_frames);
            roll_rows(&s, split, tmp);
        }
        backward = !backward;
    }
    /* LastPrism */
    run_phase(&s, PH_XB, start, gts, 0);
    run_phase(&s, PH_DOWN, start, gts, 1);
    gts += s.mpss;
    if (backward) {
        roll_rows(&s, -split, tmp);
        nframes = window_write(&s, gts, sub, frames, nframes, max_frames);
    } else {
        nframes = window_write(&s, gts, sub, frames, nframes, max_frames);
        roll_rows(&s, split, tmp);
    }
    if (final_out) {
        /* After the last write the window has slid and the last completed
         * level sits at index its-1.  A final sendForward leaves the rows
         * rolled by bs/2, so undo that before copying out. */
        if (!backward)
            roll_rows(&s, -split, tmp);
        memcpy(final_out, s.W + (long)(its - 1) * plane, sizeof(double) * plane);
    }
    free(tmp);
    free(s.W);
    return nframes;
}

int oracle_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------ heat, float32 -- */
/* The reference run with `dtype: float32` (io.py:72-73) keeps every level in
 * a float32 array, but heat.py's courant (heat.py:37) is a float64 scalar, so
 * numpy evaluates each step in float64 and rounds the result to float32 when
 * it is stored: u_{n+1} = float32(heat_fe_64(u_n)).  Forward Euler only.
 * Pinned against the reference's float32 standard frames
 * (tests/golden/heat_fe_f32_*.npz). */
long oracle_heat_f32(float *u, int nx, int ny, double courant, long nlevels, int nthreads)
{
    size_t n = (size_t)nx * ny;
    float *tmp = (float *)malloc(n * sizeof(float));
    if (!tmp) return -1;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    for (long L = 0; L < nlevels; ++L) {
#pragma omp parallel for schedule(static)
        for (int x = 0; x < nx; ++x) {
            const float *r = u + (size_t)x * ny;
            const float *up = u + (size_t)((x + nx - 1) % nx) * ny;
            const float *dn = u + (size_t)((x + 1) % nx) * ny;
            for (int y = 0; y < ny; ++y) {
                double c = r[y];
                double dx2 = courant * (((double)dn[y] - 2.0 * c) + (double)up[y]);
                double dy2 = courant * (((double)r[(y + 1) % ny] - 2.0 * c) + (double)r[(y + ny - 1) % ny]);
                tmp[(size_t)x * ny + y] = (float)((dx2 + dy2) + c);
            }
        }
        memcpy(u, tmp, n * sizeof(float));
    }
    free(tmp);
    return nlevels;
}
