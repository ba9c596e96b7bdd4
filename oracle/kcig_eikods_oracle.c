/* CPU restatement of eikods2d's table computation -- TEST INFRASTRUCTURE ONLY
 * (used by tests/ as the checker of the GPU table generator, never by the
 * library).  Two solvers of the same local problem on a 2-D grid:
 *
 *   method 0 (marching): fast marching as eikods2d runs it
 *     (SERECKIRCH/src/eikods.cpp:66-111, neighbors.cpp:34-52, 74-88, 106-188,
 *     271-302, 330-342, 418-484, pqueue.cpp:24-85): the same source box, the
 *     same binary heap (which is not re-sifted when a queued value drops), the
 *     same upwind quadratic in double precision and the same stopping rule
 *     (the loop ends once every point has been reached, leaving the last
 *     front at its tentative values).  Pinned bit-exact to the reference
 *     eikods2d on the committed fixtures.
 *   method 1 (sweeps): Gauss-Seidel sweeps in the four diagonal orderings
 *     with the same local update until four consecutive sweeps change nothing
 *     -- the fixed point the GPU kernels compute, sweep for sweep.
 *
 * Both then take the source-position derivatives in order of increasing time
 * (eikods.cpp:119-211, eikods_dt / eikods_dt1) and, on request, the
 * branch-aware gradients of src/eikods2d.cpp:30-68.  Every expression keeps
 * the reference's types and evaluation order (the reference build is x86-64
 * SSE without FMA; build this file with -ffp-contract=off).
 */
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

enum { ST_IN = 0, ST_FRONT = 1, ST_OUT = 2 };

typedef struct {
    int nz, nx;       /* grid: depth fastest */
    float d[3];       /* sampling: depth, lateral, third axis */
    float rdx[2];     /* 1/d^2 rounded to float */
    int order;
    const float *vv;  /* slowness squared */
    float *t;         /* traveltime being built */
    int *state;       /* marching status */
    int use_state;    /* 1: marching (status checks), 0: sweeps */
    float **heap;     /* 1-based binary heap of pointers into t */
    int hn;           /* heap size */
} Grid;

/* ------------------------------------------------------------ heap -- */

static void heap_push(Grid *g, float *v)
{
    int q = ++g->hn;
    g->heap[q] = v;
    /* move up while the parent is not smaller (pqueue.cpp:24-40) */
    for (int p = q >> 1; p > 0; p >>= 1) {
        if (*v > *g->heap[p]) break;
        g->heap[q] = g->heap[p];
        q = p;
    }
    g->heap[q] = v;
}

static float *heap_pop(Grid *g)
{
    if (g->hn < 1) return NULL;
    float *top = g->heap[1];
    float *last = g->heap[g->hn--];
    const int n = g->hn;
    int q = 1;
    for (int c = 2; c <= n; c <<= 1) {
        if (c < n && *g->heap[c] > *g->heap[c + 1]) c++;
        if (*last <= *g->heap[c]) break;
        g->heap[q] = g->heap[c];
        q = c;
    }
    g->heap[q] = last;
    return top;
}

/* ---------------------------------------------------- local update -- */

typedef struct {
    double stencil, value, delta;
} Axis;

static void axis_setup(const Grid *g, Axis *x, int i, int ii, int n, int s, float rdx)
{
    const float a = ii > 0 ? g->t[i - s] : FLT_MAX;
    const float b = ii < n - 1 ? g->t[i + s] : FLT_MAX;
    x->delta = rdx;
    x->stencil = x->value = (a < b) ? a : b;
    if (g->order > 1) {
        float t2;
        if (a < b && ii - 2 >= 0) {
            const int k = i - 2 * s;
            if ((!g->use_state || g->state[k] != ST_OUT) && a >= (t2 = g->t[k])) {
                x->delta *= 2.25;
                x->stencil = (4.0 * x->value - t2) / 3.0;
            }
        }
        if (a > b && ii + 2 <= n - 1) {
            const int k = i + 2 * s;
            if ((!g->use_state || g->state[k] != ST_OUT) && b >= (t2 = g->t[k])) {
                x->delta *= 2.25;
                x->stencil = (4.0 * x->value - t2) / 3.0;
            }
        }
    }
}

/* root of sum over the first m axes of delta (t - stencil)^2 = v1 */
static int solve_axes(int m, Axis *const *v, double v1, float *res)
{
    double a = 0.0, b = 0.0, c = 0.0;
    for (int j = 0; j < m; j++) {
        a += v[j]->delta;
        b += v[j]->stencil * v[j]->delta;
        c += v[j]->stencil * v[j]->stencil * v[j]->delta;
    }
    b /= a;
    const double discr = b * b + (v1 - c) / a;
    if (discr < 0.0) return 0;
    const double t = b + sqrt(discr);
    if (t <= v[m - 1]->value) return 0;
    *res = (float)t;
    return 1;
}

static float local_time(const Grid *g, int i)
{
    Axis x[3];
    const int iz = i % g->nz, ix = i / g->nz;
    axis_setup(g, &x[0], i, iz, g->nz, 1, g->rdx[0]);
    axis_setup(g, &x[1], i, ix, g->nx, g->nz, g->rdx[1]);
    x[2].delta = 0.0; /* the third axis of a 2-D grid: never reached */
    x[2].stencil = x[2].value = FLT_MAX;
    /* ascending order of value with the marching code's tie rules */
    Axis *v[3];
    if (x[0].value <= x[1].value) {
        if (x[1].value <= x[2].value) { v[0] = &x[0]; v[1] = &x[1]; v[2] = &x[2]; }
        else if (x[2].value <= x[0].value) { v[0] = &x[2]; v[1] = &x[0]; v[2] = &x[1]; }
        else { v[0] = &x[0]; v[1] = &x[2]; v[2] = &x[1]; }
    } else {
        if (x[0].value <= x[2].value) { v[0] = &x[1]; v[1] = &x[0]; v[2] = &x[2]; }
        else if (x[2].value <= x[1].value) { v[0] = &x[2]; v[1] = &x[1]; v[2] = &x[0]; }
        else { v[0] = &x[1]; v[1] = &x[2]; v[2] = &x[0]; }
    }
    const double v1 = g->vv[i];
    float r;
    if (v[2]->value < FLT_MAX) {
        if (solve_axes(3, v, v1, &r) || solve_axes(2, v, v1, &r) || solve_axes(1, v, v1, &r)) return r;
    } else if (v[1]->value < FLT_MAX) {
        if (solve_axes(2, v, v1, &r) || solve_axes(1, v, v1, &r)) return r;
    } else if (v[0]->value < FLT_MAX) {
        if (solve_axes(1, v, v1, &r)) return r;
    }
    return FLT_MAX;
}

/* --------------------------------------------------------- source -- */

/* The box of (2 b + 1)^2 samples around the source at straight-ray times
 * with the slowness of the box centre; returns the number of points left
 * and marks the box in `inbox` (may be NULL). */
static int source_box(Grid *g, const float xs[3], int b1, int b2, unsigned char *inbox)
{
    const int n[3] = {g->nz, g->nx, 1}, b[2] = {b1, b2};
    const int ntot = g->nz * g->nx;
    int st[3], en[3];
    for (int i = 0; i < ntot; i++) {
        g->state[i] = ST_OUT;
        g->t[i] = FLT_MAX;
        if (inbox) inbox[i] = 0;
    }
    for (int j = 0; j < 2; j++) {
        const int is = xs[j] / g->d[j] + 0.5;
        st[j] = is - b[j];
        en[j] = is + b[j];
        if (st[j] < 0) st[j] = 0; else if (st[j] >= n[j]) st[j] = n[j] - 1;
        if (en[j] < 0) en[j] = 0; else if (en[j] >= n[j]) en[j] = n[j] - 1;
    }
    st[2] = en[2] = 0; /* the third axis has one sample */
    const int ic = (st[0] + en[0]) / 2 + n[0] * ((st[1] + en[1]) / 2 + n[1] * (st[2] + en[2]) / 2);
    const double v1 = g->vv[ic];
    int left = ntot;
    for (int iy = st[1]; iy <= en[1]; iy++) {
        for (int iz = st[0]; iz <= en[0]; iz++) {
            left--;
            const int i = iz + n[0] * iy;
            double e[3];
            e[0] = xs[0] - iz * g->d[0];
            e[1] = xs[1] - iy * g->d[1];
            e[2] = xs[2] - 0 * g->d[2];
            double d2 = 0.0;
            for (int j = 0; j < 3; j++) d2 += e[j] * e[j];
            g->t[i] = sqrtf(v1 * d2);
            g->state[i] = ST_IN;
            if (inbox) inbox[i] = 1;
            if (g->heap && ((n[0] > 1 && (iz == st[0] || iz == en[0])) || (n[1] > 1 && (iy == st[1] || iy == en[1]))))
                heap_push(g, g->t + i);
        }
    }
    return left;
}

/* --------------------------------------------------------- solvers -- */

static int relax(Grid *g, int k)
{
    const float value = local_time(g, k);
    if (value < g->t[k]) {
        g->t[k] = value;
        if (g->state[k] == ST_OUT) {
            g->state[k] = ST_FRONT;
            heap_push(g, g->t + k);
            return 1;
        }
    }
    return 0;
}

static int relax_neighbours(Grid *g, int i)
{
    const int iz = i % g->nz, ix = i / g->nz;
    const int ii[2] = {iz, ix}, n[2] = {g->nz, g->nx}, s[2] = {1, g->nz};
    int added = 0;
    for (int j = 0; j < 2; j++) {
        if (ii[j] + 1 <= n[j] - 1 && g->state[i + s[j]] != ST_IN) added += relax(g, i + s[j]);
        if (ii[j] - 1 >= 0 && g->state[i - s[j]] != ST_IN) added += relax(g, i - s[j]);
    }
    return added;
}

static void march(Grid *g, const float xs[3], int b1, int b2)
{
    g->use_state = 1;
    g->hn = 0;
    int left = source_box(g, xs, b1, b2, NULL);
    while (left > 0) {
        float *p = heap_pop(g);
        if (!p) break;
        const int i = (int)(p - g->t);
        g->state[i] = ST_IN;
        left -= relax_neighbours(g, i);
    }
}

static int sweep_fixed_point(Grid *g, const float xs[3], int b1, int b2, int max_iter, unsigned char *inbox)
{
    float **heap = g->heap;
    g->heap = NULL;
    source_box(g, xs, b1, b2, inbox);
    g->heap = heap;
    g->use_state = 0;
    int quiet = 0;
    for (int sweep = 0; sweep < 4 * max_iter; sweep++) {
        const int dir = sweep & 3, fz = (dir & 1) == 0, fx = (dir & 2) == 0;
        int changed = 0;
        for (int u = 0; u < g->nx; u++) {
            for (int w = 0; w < g->nz; w++) {
                const int ix = fx ? u : g->nx - 1 - u, iz = fz ? w : g->nz - 1 - w;
                const int i = iz + g->nz * ix;
                if (inbox[i]) continue;
                const float q = local_time(g, i);
                if (q < g->t[i]) {
                    g->t[i] = q;
                    changed = 1;
                }
            }
        }
        quiet = changed ? 0 : quiet + 1;
        if (quiet >= 4) return sweep + 1;
    }
    return 0;
}

/* ------------------------------------------------- source derivative -- */

static const float *g_sort_t;
static int by_time(const void *a, const void *b)
{
    const float ta = g_sort_t[*(const int *)a], tb = g_sort_t[*(const int *)b];
    if (ta > tb) return 1;
    if (ta == tb) return 0;
    return -1;
}

/* eikods_dt1 for point i0: l = perturbation axis (0 depth, 1 lateral) */
static void deriv_point(const Grid *g, int l, int i0, float *dl1, float *ds1)
{
    const float *t0 = g->t, *v0 = g->vv;
    const int n[2] = {g->nz, g->nx}, s[2] = {1, g->nz};
    const int ii[2] = {i0 % g->nz, i0 / g->nz};
    double rhs = 0.0, den = 0.0, dw = 0.0, dt = 0.0;
    for (int j = 0; j < 2; j++) {
        const int a = i0 - s[j], b = i0 + s[j];
        int i1;
        if (ii[j] == 0 || (ii[j] != n[j] - 1 && t0[a] > t0[b])) i1 = b;
        else i1 = a;
        if (t0[i1] < t0[i0]) {
            rhs += (t0[i0] - t0[i1]) * dl1[i1] / (g->d[j] * g->d[j]);
            den += (t0[i0] - t0[i1]) / (g->d[j] * g->d[j]);
            if (l == j) {
                if (i1 == b) {
                    const int i2 = i1 + s[j];
                    if (ii[j] < n[j] - 2 && t0[i1] > t0[i2])
                        dt = (-t0[i2] + 4. * t0[i1] - 3. * t0[i0]) / (2. * g->d[j]);
                    else
                        dt = (t0[i1] - t0[i0]) / g->d[j];
                } else {
                    const int i2 = i1 - s[j];
                    if (ii[j] > 1 && t0[i1] > t0[i2])
                        dt = (3. * t0[i0] - 4. * t0[i1] + t0[i2]) / (2. * g->d[j]);
                    else
                        dt = (t0[i0] - t0[i1]) / g->d[j];
                }
            }
        }
    }
    if (den == 0.0) {
        dl1[i0] = 0.0f;
        ds1[i0] = 0.0f;
        return;
    }
    const int sl = s[l];
    if (0 < ii[l] && ii[l] < n[l] - 1)
        dw = (v0[i0 + sl] - v0[i0 - sl]) / (2. * g->d[l]);
    else if (ii[l] == 0)
        dw = (-v0[i0 + 2 * sl] + 4. * v0[i0 + sl] - 3. * v0[i0]) / (2. * g->d[l]);
    else
        dw = (3. * v0[i0] - 4. * v0[i0 - sl] + v0[i0 - 2 * sl]) / (2. * g->d[l]);
    dl1[i0] = (0.5 * dw + rhs) / den;
    ds1[i0] = dl1[i0] - dt;
}

static void derivatives(const Grid *g, int l, float *dl1, float *ds1)
{
    const int ntot = g->nz * g->nx;
    int *order = malloc(sizeof(int) * ntot);
    for (int i = 0; i < ntot; i++) order[i] = i;
    g_sort_t = g->t;
    qsort(order, ntot, sizeof(int), by_time);
    for (int k = 0; k < ntot; k++) deriv_point(g, l, order[k], dl1, ds1);
    free(order);
}

/* ---------------------------------------------- upwind gradients -- */

static float upwind(const float *t, int i0, int ii, int n, int s, float dd)
{
    const int a = i0 - s, b = i0 + s;
    int i1;
    if (ii == 0) i1 = b;
    else if (ii != n - 1 && t[b] < t[a]) i1 = b;
    else i1 = a;
    if (!(t[i1] < t[i0])) return 0.0f;
    if (i1 == b) {
        const int i2 = i1 + s;
        if (ii < n - 2 && t[i2] < t[i1]) return (-t[i2] + 4.0f * t[i1] - 3.0f * t[i0]) / (2.0f * dd);
        return (t[i1] - t[i0]) / dd;
    }
    const int i2 = i1 - s;
    if (ii > 1 && t[i2] < t[i1]) return (3.0f * t[i0] - 4.0f * t[i1] + t[i2]) / (2.0f * dd);
    return (t[i0] - t[i1]) / dd;
}

void oracle_upwind_grads(int nz, int nx, float dz, float dx, const float *t, float *gz, float *gx)
{
    for (int i = 0; i < nz * nx; i++) {
        if (gz) gz[i] = upwind(t, i, i % nz, nz, 1, dz);
        if (gx) gx[i] = upwind(t, i, i / nz, nx, nz, dx);
    }
}

/* ------------------------------------------------------ entry point -- */

/* method 0: marching (eikods2d), 1: sweeps to the fixed point.  vel [nx][nz]
 * (velocity, or slowness squared when vel_is_s2), shots [nshot][3] (depth,
 * lateral, third axis), outputs [nshot][nx][nz] (dl1/ds1/gz/gx may be NULL;
 * sweeps [nshot] may be NULL).  Returns 0, or -1 on bad arguments, -2 when
 * the sweeps found no fixed point within max_iter. */
int oracle_eikods(int method, int nz, int nx, float o1, float o2, float d1, float d2, float o3, float d3,
                  const float *vel, int vel_is_s2, const float *shots, int nshot, int b1, int b2, int order, int l,
                  int max_iter, float *t, float *dl1, float *ds1, float *gz, float *gx, int *sweeps)
{
    if (nz < 3 || nx < 3 || nshot < 1 || (order != 1 && order != 2) || (l != 0 && l != 1)) return -1;
    const int ntot = nz * nx;
    float *vv = malloc(sizeof(float) * ntot);
    for (int i = 0; i < ntot; i++) {
        const float v = vel[i];
        vv[i] = vel_is_s2 ? v : 1. / (v * v);
    }
    Grid g;
    memset(&g, 0, sizeof(g));
    g.nz = nz;
    g.nx = nx;
    g.d[0] = d1;
    g.d[1] = d2;
    g.d[2] = d3;
    g.rdx[0] = 1. / (d1 * d1);
    g.rdx[1] = 1. / (d2 * d2);
    g.order = order;
    g.vv = vv;
    g.state = malloc(sizeof(int) * ntot);
    g.heap = calloc((size_t)ntot + 2, sizeof(float *)); /* every point enters at most once */
    unsigned char *inbox = malloc(ntot);
    float *tdl = malloc(sizeof(float) * ntot), *tds = malloc(sizeof(float) * ntot);
    int rc = 0;
    if (b1 < 1) b1 = 1;
    if (b2 < 1) b2 = 1;
    for (int js = 0; js < nshot; js++) {
        const float xs[3] = {shots[3 * js] - o1, shots[3 * js + 1] - o2, shots[3 * js + 2] - o3};
        g.t = t + (size_t)js * ntot;
        int ns = 0;
        if (method == 0) {
            march(&g, xs, b1, b2);
        } else {
            ns = sweep_fixed_point(&g, xs, b1, b2, max_iter, inbox);
            if (ns == 0) rc = -2;
        }
        if (sweeps) sweeps[js] = ns;
        if (dl1 || ds1) {
            derivatives(&g, l, tdl, tds);
            if (dl1) memcpy(dl1 + (size_t)js * ntot, tdl, sizeof(float) * ntot);
            if (ds1) memcpy(ds1 + (size_t)js * ntot, tds, sizeof(float) * ntot);
        }
        if (gz || gx)
            oracle_upwind_grads(nz, nx, d1, d2, g.t, gz ? gz + (size_t)js * ntot : NULL,
                                gx ? gx + (size_t)js * ntot : NULL);
    }
    free(vv);
    free(g.state);
    free(g.heap);
    free(inbox);
    free(tdl);
    free(tds);
    return rc;
}
