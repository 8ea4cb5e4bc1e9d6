/*
 * ORACLE -- test infrastructure only.  A plain-C restatement of the reference's CPU certificate for the whole-cell
 * Jacobian-determinant proof of a Q1 displacement field.  Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg use it, as the checker; the product path never calls it.
 *
 * Parity is pinned by tests/golden/certificate.npz and tests/golden/cells.npz, generated by running the reference
 * (tests/golden/make_golden.py).  Every function names the reference function it restates (paths inside the
 * reference project, jd_curl/three_d/...).
 *
 * Arithmetic contract (the reference's): IEEE binary64, round to nearest, no contraction (build with
 * -ffp-contract=off), IEEE division; every interval operation rounds to nearest and then steps one ulp outward with
 * libm nextafter (interval.py:52 Interval.outward, compiled_enclosure.py:163 _nr_outward).  min/max follow Numba's
 * scalar np.minimum/np.maximum: the first operand when a <= b (a >= b) or when a is NaN, else the second.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>


/* ------------------------------------------------------------------ interval primitives (compiled_enclosure.py) */
static inline double nmin(double a, double b) { return (a <= b || a != a) ? a : b; }
static inline double nmax(double a, double b) { return (a >= b || a != a) ? a : b; }
static inline int fin(double x) { return isfinite(x) != 0; }

/* _nr_outward (compiled_enclosure.py:163): outward step, validity = both finite and lo <= hi */
static inline int out_(double lo, double hi, double *rl, double *rh) {
    lo = nextafter(lo, -INFINITY);
    hi = nextafter(hi, INFINITY);
    *rl = lo; *rh = hi;
    return fin(lo) && fin(hi) && lo <= hi;
}
static inline int add_(double al, double ah, double bl, double bh, double *rl, double *rh) {
    return out_(al + bl, ah + bh, rl, rh);
}
static inline int sub_(double al, double ah, double bl, double bh, double *rl, double *rh) {
    return out_(al - bh, ah - bl, rl, rh);
}
/* _nr_mul (compiled_enclosure.py:179): four rounded products, ordered min/max, outward */
static inline int mul_(double al, double ah, double bl, double bh, double *rl, double *rh) {
    double x = al * bl, y = al * bh, z = ah * bl, w = ah * bh;
    return out_(nmin(nmin(nmin(x, y), z), w), nmax(nmax(nmax(x, y), z), w), rl, rh);
}

/* left-associated cofactor expansion shared by every interval kernel (compiled_enclosure.py:70 _determinant_bounds,
 * and the same sequence inside _chunk_hoisted_margins :234-248 and _fallback_kernel) */
static inline int det_(const double fl[3][3], const double fh[3][3], double *jl, double *jh) {
    double p1l, p1h, p2l, p2h, al, ah, bl, bh, cl, ch, t1l, t1h, t2l, t2h, sl, sh, t3l, t3h;
    int ok = 1;
    ok &= mul_(fl[1][1], fh[1][1], fl[2][2], fh[2][2], &p1l, &p1h);
    ok &= mul_(fl[1][2], fh[1][2], fl[2][1], fh[2][1], &p2l, &p2h);
    ok &= sub_(p1l, p1h, p2l, p2h, &al, &ah);
    ok &= mul_(fl[1][2], fh[1][2], fl[2][0], fh[2][0], &p1l, &p1h);
    ok &= mul_(fl[1][0], fh[1][0], fl[2][2], fh[2][2], &p2l, &p2h);
    ok &= sub_(p1l, p1h, p2l, p2h, &bl, &bh);
    ok &= mul_(fl[1][0], fh[1][0], fl[2][1], fh[2][1], &p1l, &p1h);
    ok &= mul_(fl[1][1], fh[1][1], fl[2][0], fh[2][0], &p2l, &p2h);
    ok &= sub_(p1l, p1h, p2l, p2h, &cl, &ch);
    ok &= mul_(fl[0][0], fh[0][0], al, ah, &t1l, &t1h);
    ok &= mul_(fl[0][1], fh[0][1], bl, bh, &t2l, &t2h);
    ok &= add_(t1l, t1h, t2l, t2h, &sl, &sh);
    ok &= mul_(fl[0][2], fh[0][2], cl, ch, &t3l, &t3h);
    ok &= add_(sl, sh, t3l, t3h, jl, jh);
    return ok;
}

/* vertex a = x + 2y + 4z of cell (x0,y0,z0): node offset in a (nz,ny,nx) C-order grid (cell_q1.py:10 VERTICES) */
static inline int64_t vnode(int64_t base, int a, int64_t ny, int64_t nx) {
    return base + (int64_t)(a >> 2) * ny * nx + (int64_t)((a >> 1) & 1) * nx + (a & 1);
}

/* ------------------------------------------------------------------ edge hull (compiled_enclosure.py:210) */
/* _nr_entry (compiled_enclosure.py:186): F_rj interval of one cell from the hull of 4 edge differences */
static inline int entry_(const double *u, int64_t base, int64_t ny, int64_t nx, int j, int r, double h,
                         double *lo, double *hi) {
    int ok = 1;
    double lower = INFINITY, upper = -INFINITY;
    for (int a = 0; a < 8; a++) {
        if (a & (1 << j)) continue;
        int b = a | (1 << j);
        double d = u[3 * vnode(base, b, ny, nx) + r] - u[3 * vnode(base, a, ny, nx) + r];
        if (!fin(d)) ok = 0;
        lower = nmin(lower, d);
        upper = nmax(upper, d);
    }
    double l, hh;
    ok &= out_(lower, upper, &l, &hh);
    ok &= out_(l / h, hh / h, &l, &hh);
    double id = (r == j) ? 1.0 : 0.0;
    ok &= add_(l, hh, id, id, lo, hi);
    return ok;
}

/* cells [start, stop) of the grid; the caller splits the range over threads */
void oc_edge_hull(const double *u, int64_t nz, int64_t ny, int64_t nx, const double *h, double delta,
                  int64_t start, int64_t stop, double *margin, uint8_t *flag) {
    int64_t cy = ny - 1, cx = nx - 1;
    (void)nz;
    for (int64_t c = start; c < stop; c++) {
        int64_t x0 = c % cx, y0 = (c / cx) % cy, z0 = c / (cx * cy);
        int64_t base = (z0 * ny + y0) * nx + x0;
        double fl[3][3], fh[3][3];
        int ok = 1;
        for (int j = 0; j < 3; j++)           /* legacy (j outer, r inner) evaluation order */
            for (int r = 0; r < 3; r++)
                ok &= entry_(u, base, ny, nx, j, r, h[j], &fl[r][j], &fh[r][j]);
        double jl, jh, ml, mh;
        ok &= det_(fl, fh, &jl, &jh);
        ok &= out_(jl - delta, jh - delta, &ml, &mh);   /* Interval.__sub__(point delta) */
        margin[c] = ml;
        flag[c] = ok ? 0 : 1;
    }
}

/* ------------------------------------------------------------------ prescreen (certificate_prescreen.py:66-122) */
void oc_prescreen(const double *u, int64_t nz, int64_t ny, int64_t nx, const double *D /* (3,27,8) */,
                  const int64_t *cells, int64_t start, int64_t stop, double g12, double g6, double g3, double sq27,
                  double eta, double *out) {
    int64_t cy = ny - 1, cx = nx - 1;
    (void)nz;
    int64_t off[8];
    for (int a = 0; a < 8; a++) off[a] = (int64_t)(a >> 2) * ny * nx + (int64_t)((a >> 1) & 1) * nx + (a & 1);
    for (int64_t i = start; i < stop; i++) {
        int64_t c = cells[i];
        int64_t x0 = c % cx, y0 = (c / cx) % cy, z0 = c / (cx * cy);
        int64_t base = (z0 * ny + y0) * nx + x0;
        double b[27], F[3][3];
        double sigma = 0., phi = 0., big = 0.;
        int finite = 1;
        for (int p = 0; p < 27; p++) {
            for (int r = 0; r < 3; r++) {
                for (int j = 0; j < 3; j++) {
                    double acc = 0., mag = 0.;
                    for (int a = 0; a < 8; a++) {
                        double term = u[3 * (base + off[a]) + r] * D[(j * 27 + p) * 8 + a];
                        acc += term;
                        mag += fabs(term);
                    }
                    F[r][j] = acc;
                    if (mag > sigma) sigma = mag;
                }
                F[r][r] += 1.;
            }
            for (int r = 0; r < 3; r++)
                for (int j = 0; j < 3; j++)
                    if (fabs(F[r][j]) > phi) phi = fabs(F[r][j]);
            double v = F[0][0] * (F[1][1] * F[2][2] - F[1][2] * F[2][1])
                     + F[0][1] * (F[1][2] * F[2][0] - F[1][0] * F[2][2])
                     + F[0][2] * (F[1][0] * F[2][1] - F[1][1] * F[2][0]);
            b[p] = v;
            if (fabs(v) > big) big = fabs(v);
        }
        static const int strides[3] = {1, 3, 9};
        for (int s = 0; s < 3; s++) {
            int stride = strides[s];
            for (int p = 0; p < 27; p++)
                if ((p / stride) % 3 == 1) b[p] = 2. * b[p] - .5 * (b[p - stride] + b[p + stride]);
        }
        double e = g12 * (sigma + phi) + eta;
        double P = phi + e;
        double ej = sq27 * e * (3. * P * P + 3. * P * e + e * e) + 6. * g6 * P * P * P;
        double bound = 1.01 * (27. * ej + 135. * g3 * big) + eta;
        double low = INFINITY;
        for (int p = 0; p < 27; p++) {
            double w = b[p];
            if (!(w == w) || w == INFINITY || w == -INFINITY) finite = 0;
            else if (w < low) low = w;
        }
        if (!(bound == bound) || bound == INFINITY || !(sigma == sigma) || sigma == INFINITY) finite = 0;
        out[i] = finite ? low - bound : NAN;
    }
}

/* ------------------------------------------------------------------ fallback arrays (compiled_fallback.py:63-174) */
/* edge tables in jacobian_intervals' loop order (compiled_fallback.py:191 _edge_tables) */
static int g_pairs[3][4][2];
static double g_weights[3][4][27];
static int g_tables_ready = 0;

static void tables_(void) {
    if (g_tables_ready) return;
    static const double pts[3] = {0., .5, 1.};
    for (int j = 0; j < 3; j++) {
        int e = 0;
        for (int a = 0; a < 8; a++) {
            int bits[3] = {a & 1, (a >> 1) & 1, (a >> 2) & 1};
            if (bits[j]) continue;
            int b = a | (1 << j);
            for (int p = 0; p < 27; p++) {
                double coord[3] = {pts[p % 3], pts[(p / 3) % 3], pts[p / 9]};
                double w = 1.;
                for (int k = 0; k < 3; k++) {
                    if (k == j) continue;
                    w *= bits[k] ? coord[k] : 1 - coord[k];
                }
                g_weights[j][e][p] = w;
            }
            g_pairs[j][e][0] = a; g_pairs[j][e][1] = b;
            e++;
        }
    }
    g_tables_ready = 1;
}

/* one cell: v = (8,3) vertex displacements; outputs 27 each; returns 1 iff every interval/sample is finite */
int oc_fallback_cell(const double *v, const double *spacing, double delta, double *plo, double *phi, double *clo,
                     double *chi, double *samples) {
    tables_();
    int ok = 1;
    double flo[27][3][3], fhi[27][3][3], elo[4][3], ehi[4][3], blo[27], bhi[27], fs[27][3][3];
    for (int j = 0; j < 3; j++) {
        double h = spacing[j];
        for (int e = 0; e < 4; e++) {
            int a = g_pairs[j][e][0], b = g_pairs[j][e][1];
            for (int r = 0; r < 3; r++) {
                double d = v[3 * b + r] - v[3 * a + r];
                double sl, sh, ql, qh;
                ok &= out_(d, d, &sl, &sh);                          /* point - point */
                double x1 = sl / h, x2 = sh / h;                     /* interval / point h */
                ok &= out_(nmin(nmin(nmin(x1, x1), x2), x2), nmax(nmax(nmax(x1, x1), x2), x2), &ql, &qh);
                elo[e][r] = ql; ehi[e][r] = qh;
            }
        }
        for (int p = 0; p < 27; p++)
            for (int r = 0; r < 3; r++) {
                double dl = 0., dh = 0.;
                for (int e = 0; e < 4; e++) {
                    double w = g_weights[j][e][p], wl, wh;
                    ok &= out_(elo[e][r] * w, ehi[e][r] * w, &wl, &wh);
                    ok &= add_(dl, dh, wl, wh, &dl, &dh);
                }
                double c = (r == j) ? 1. : 0.;
                ok &= add_(dl, dh, c, c, &flo[p][r][j], &fhi[p][r][j]);
            }
    }
    for (int p = 0; p < 27; p++) {
        double jl, jh, ml, mh;
        ok &= det_((const double(*)[3])flo[p], (const double(*)[3])fhi[p], &jl, &jh);
        ok &= sub_(jl, jh, delta, delta, &ml, &mh);                  /* "- delta" */
        plo[p] = ml; phi[p] = mh;
        blo[p] = ml; bhi[p] = mh;
    }
    /* lagrange_to_bernstein: storage index 9*iz+3*iy+ix; axes x, then y, then z */
    static const int plan[3][5] = {{1, 3, 9, 3, 3}, {3, 3, 9, 3, 1}, {9, 3, 3, 3, 1}};
    for (int s = 0; s < 3; s++) {
        int stride = plan[s][0], o1 = plan[s][1], s1 = plan[s][2], o2 = plan[s][3], s2 = plan[s][4];
        for (int i1 = 0; i1 < o1; i1++)
            for (int i2 = 0; i2 < o2; i2++) {
                int i0 = i1 * s1 + i2 * s2, a0 = i0, a1 = i0 + stride, a2 = i0 + 2 * stride;
                double ml1, mh1, sl1, sh1, hl1, hh1, nl, nh;
                ok &= mul_(blo[a1], bhi[a1], 2., 2., &ml1, &mh1);
                ok &= add_(blo[a0], bhi[a0], blo[a2], bhi[a2], &sl1, &sh1);
                ok &= mul_(sl1, sh1, .5, .5, &hl1, &hh1);
                ok &= sub_(ml1, mh1, hl1, hh1, &nl, &nh);
                blo[a1] = nl; bhi[a1] = nh;
            }
    }
    for (int p = 0; p < 27; p++) { clo[p] = blo[p]; chi[p] = bhi[p]; }
    /* _sample_jacobians (float64 diagnostic) */
    for (int p = 0; p < 27; p++)
        for (int r = 0; r < 3; r++)
            for (int j = 0; j < 3; j++) fs[p][r][j] = (r == j) ? 1. : 0.;
    for (int j = 0; j < 3; j++) {
        double h = spacing[j];
        for (int e = 0; e < 4; e++) {
            int a = g_pairs[j][e][0], b = g_pairs[j][e][1];
            for (int p = 0; p < 27; p++) {
                double w = g_weights[j][e][p];
                for (int r = 0; r < 3; r++) fs[p][r][j] = fs[p][r][j] + ((v[3 * b + r] - v[3 * a + r]) / h) * w;
            }
        }
    }
    for (int p = 0; p < 27; p++) {
        int finite = 1;
        for (int r = 0; r < 3; r++)
            for (int j = 0; j < 3; j++) finite = finite && fin(fs[p][r][j]);
        double (*f)[3] = fs[p];
        double a00 = f[1][1] * f[2][2] - f[1][2] * f[2][1];
        double a01 = f[1][2] * f[2][0] - f[1][0] * f[2][2];
        double a02 = f[1][0] * f[2][1] - f[1][1] * f[2][0];
        double a10 = f[2][1] * f[0][2] - f[2][2] * f[0][1];
        double a11 = f[2][2] * f[0][0] - f[2][0] * f[0][2];
        double a12 = f[2][0] * f[0][1] - f[2][1] * f[0][0];
        double a20 = f[0][1] * f[1][2] - f[0][2] * f[1][1];
        double a21 = f[0][2] * f[1][0] - f[0][0] * f[1][2];
        double a22 = f[0][0] * f[1][1] - f[0][1] * f[1][0];
        double all9[9] = {a00, a01, a02, a10, a11, a12, a20, a21, a22};
        for (int k = 0; k < 9; k++) finite = finite && fin(all9[k]);
        double t0 = f[0][0] * a00, t1 = f[0][1] * a01, t2 = f[0][2] * a02;
        double s = 0.;
        s += t0; s += t1; s += t2;
        finite = finite && fin(t0) && fin(t1) && fin(t2) && fin(s);
        samples[p] = s;
        ok = ok && finite;
    }
    return ok;
}

/* ------------------------------------------------------------------ subdivision (feasibility.py:295 _classify) */
enum { ST_FEASIBLE = 0, ST_INFEASIBLE = 1, ST_UNCERTAIN = 2 };
/* reason codes: the index in tests/golden REASONS */
enum { R_ENCLOSURE = 0, R_BERNSTEIN = 1, R_VIOLATION = 2, R_ARITH = 3, R_SUBDIV_BUDGET = 4, R_NONFINITE = 5,
       R_BOUNDARY = 6, R_DOMAIN = 7, R_UNSUPPORTED = 8, R_SAMPLE_WITNESS = 9, R_SUBDIV_WITNESS = 10,
       R_BOX_BUDGET = 11, R_DEPTH_BUDGET = 12 };

typedef struct {
    double lo[27], hi[27];
    double low[3], high[3];
    int depth;
    double key;
    int64_t serial;
} box_t;

typedef struct {
    int32_t status, reason, has_margin, has_witness;
    int64_t boxes, depth;
    double margin, witness[3];
} cls_t;

static inline int heap_less(const box_t *a, const box_t *b) {
    return a->key < b->key || (a->key == b->key && a->serial < b->serial);
}

/* result() inside _classify: margin -> (lower, margin); delta != 0 adds delta outward and may fail */
static void cls_result(cls_t *r, int status, double margin, int64_t boxes, int64_t depth, const double *w,
                       int reason, double delta) {
    r->boxes = boxes; r->depth = depth;
    if (delta != 0.) {
        double l, h;
        if (!out_(margin + delta, margin + delta, &l, &h)) {
            r->status = ST_UNCERTAIN; r->reason = R_ARITH; r->has_margin = 0; r->has_witness = 0;
            return;
        }
    }
    r->status = status; r->reason = reason; r->margin = margin; r->has_margin = 1;
    r->has_witness = w != NULL;
    if (w) { r->witness[0] = w[0]; r->witness[1] = w[1]; r->witness[2] = w[2]; }
}

static double min27(const double *x) {
    double m = x[0];
    for (int i = 1; i < 27; i++) if (x[i] < m) m = x[i];
    return m;
}

/* split_bernstein (interval.py:116) along reference axis (0=x,1=y,2=z); storage index 9*iz+3*iy+ix */
static int split_(const box_t *cur, int axis, box_t *left, box_t *right) {
    int stride = axis == 0 ? 1 : (axis == 1 ? 3 : 9);
    int ok = 1;
    for (int q = 0; q < 27; q++) {
        if (((q / stride) % 3) != 0) continue;
        int ia = q, ib = q + stride, ic = q + 2 * stride;
        double abl, abh, bcl, bch, ml, mh;
        double sl, sh;
        ok &= add_(cur->lo[ia], cur->hi[ia], cur->lo[ib], cur->hi[ib], &sl, &sh);
        ok &= mul_(sl, sh, .5, .5, &abl, &abh);
        ok &= add_(cur->lo[ib], cur->hi[ib], cur->lo[ic], cur->hi[ic], &sl, &sh);
        ok &= mul_(sl, sh, .5, .5, &bcl, &bch);
        ok &= add_(abl, abh, bcl, bch, &sl, &sh);
        ok &= mul_(sl, sh, .5, .5, &ml, &mh);
        left->lo[ia] = cur->lo[ia]; left->hi[ia] = cur->hi[ia];
        left->lo[ib] = abl; left->hi[ib] = abh;
        left->lo[ic] = ml; left->hi[ic] = mh;
        right->lo[ia] = ml; right->hi[ia] = mh;
        right->lo[ib] = bcl; right->hi[ib] = bch;
        right->lo[ic] = cur->lo[ic]; right->hi[ic] = cur->hi[ic];
    }
    return ok;
}

/* depth_first = 0: lowest-bound-first heap of (key, serial) (AdaptiveCertificateConfig, feasibility.py:319);
 * depth_first = 1: the bare CertificateConfig's pending list used as a stack (feasibility.py:326, :353-354): pop the
 * last box, push the right child and then the left one. */
void oc_classify(const double *clo, const double *chi, const double *plo, const double *phi, double delta,
                 int64_t max_depth, int64_t max_boxes, int depth_first, cls_t *res) {
    (void)plo;
    memset(res, 0, sizeof *res);
    double root_lower = min27(clo);
    /* sample witness: first (z,y,x) C-order closed27 point with p.hi <= 0 */
    for (int q = 0; q < 27; q++) {
        if (phi[q] <= 0) {
            double w[3] = {(q % 3) / 2., ((q / 3) % 3) / 2., (q / 9) / 2.};
            cls_result(res, ST_INFEASIBLE, root_lower, 1, 0, w, R_SAMPLE_WITNESS, delta);
            return;
        }
    }
    int64_t cap = max_boxes + 2;
    box_t *heap = (box_t *)malloc(sizeof(box_t) * (size_t)cap);
    int64_t nheap = 0, serial = 0, boxes = 0, depth_used = 0;
    int uncertain = 0;
    double cert_min = INFINITY;
    int have_cert = 0;
    box_t *root = &heap[nheap++];
    memcpy(root->lo, clo, sizeof root->lo); memcpy(root->hi, chi, sizeof root->hi);
    for (int k = 0; k < 3; k++) { root->low[k] = 0.; root->high[k] = 1.; }
    root->depth = 0; root->key = root_lower; root->serial = 0;
    while (nheap) {
        if (boxes >= max_boxes) {
            cls_result(res, ST_UNCERTAIN, root_lower, boxes, depth_used, NULL, R_BOX_BUDGET, delta);
            free(heap); return;
        }
        box_t cur;
        if (depth_first) {
            cur = heap[--nheap];             /* stack pop */
        } else {
            /* pop the minimum (key, serial) */
            cur = heap[0];
            heap[0] = heap[--nheap];
            for (int64_t i = 0;;) {
                int64_t l = 2 * i + 1, r = l + 1, m = i;
                if (l < nheap && heap_less(&heap[l], &heap[m])) m = l;
                if (r < nheap && heap_less(&heap[r], &heap[m])) m = r;
                if (m == i) break;
                box_t t = heap[i]; heap[i] = heap[m]; heap[m] = t; i = m;
            }
        }
        boxes += 1;
        if (cur.depth > depth_used) depth_used = cur.depth;
        double minimum = min27(cur.lo);
        if (minimum > 0) {
            if (!have_cert || minimum < cert_min) cert_min = minimum;
            have_cert = 1;
            continue;
        }
        /* corner coefficients hi[::2, ::2, ::2] in C order (iz, iy, ix) */
        int found = -1;
        for (int c = 0; c < 8 && found < 0; c++) {
            int iz = (c >> 2) & 1, iy = (c >> 1) & 1, ix = c & 1;
            if (cur.hi[9 * 2 * iz + 3 * 2 * iy + 2 * ix] <= 0) found = c;
        }
        if (found >= 0) {
            int bits[3] = {found & 1, (found >> 1) & 1, (found >> 2) & 1};   /* (ix, iy, iz) */
            double w[3];
            for (int k = 0; k < 3; k++) w[k] = bits[k] ? cur.high[k] : cur.low[k];
            cls_result(res, ST_INFEASIBLE, root_lower, boxes, depth_used, w, R_SUBDIV_WITNESS, delta);
            free(heap); return;
        }
        if (cur.depth >= max_depth) { uncertain = 1; continue; }
        int axis = 0;
        double best = cur.high[0] - cur.low[0];
        for (int k = 1; k < 3; k++) {
            double ext = cur.high[k] - cur.low[k];
            if (ext > best) { best = ext; axis = k; }
        }
        box_t left, right;
        if (!split_(&cur, axis, &left, &right)) {
            cls_result(res, ST_UNCERTAIN, root_lower, boxes, depth_used, NULL, R_ARITH, delta);
            free(heap); return;
        }
        double mid = (cur.low[axis] + cur.high[axis]) * .5;
        memcpy(left.low, cur.low, sizeof left.low); memcpy(left.high, cur.high, sizeof left.high);
        memcpy(right.low, cur.low, sizeof right.low); memcpy(right.high, cur.high, sizeof right.high);
        left.high[axis] = mid; right.low[axis] = mid;
        left.depth = right.depth = cur.depth + 1;
        if (depth_first) {                   /* stack push: right, then left (popped first) */
            heap[nheap++] = right;
            heap[nheap++] = left;
            continue;
        }
        box_t *kids[2] = {&left, &right};
        for (int k = 0; k < 2; k++) {
            serial += 1;
            kids[k]->key = min27(kids[k]->lo);
            kids[k]->serial = serial;
            int64_t i = nheap++;
            heap[i] = *kids[k];
            while (i > 0) {
                int64_t p = (i - 1) / 2;
                if (!heap_less(&heap[i], &heap[p])) break;
                box_t t = heap[i]; heap[i] = heap[p]; heap[p] = t; i = p;
            }
        }
    }
    free(heap);
    if (uncertain) { cls_result(res, ST_UNCERTAIN, root_lower, boxes, depth_used, NULL, R_DEPTH_BUDGET, delta); return; }
    cls_result(res, ST_FEASIBLE, cert_min, boxes, depth_used, NULL, R_BERNSTEIN, delta);
}

/* ------------------------------------------------------------------ certify_map (feasibility.py:393, :623) */
/* rec_i: status, reason, n_cells_checked, n_uncertain, n_infeasible, n_boxes, max_depth, witness_cell, n_fast,
 *        n_fallback, n_prescreen, has_min_jd, has_sampled_min
 * rec_f: min_jd_lower_bound, min_margin_lower_bound, sampled_min_jd, witness point xyz            */
void oc_certify_map(const double *u, int64_t nz, int64_t ny, int64_t nx, const double *spacing, const double *axx,
                    const double *axy, const double *axz, double delta, int64_t max_depth, int64_t max_boxes,
                    int64_t tile_size, const double *D, int use_prescreen, double g12, double g6, double g3,
                    double sq27, double eta, int use_hull, int depth_first, int64_t *rec_i, double *rec_f) {
    int64_t n = (nz - 1) * (ny - 1) * (nx - 1), nn = nz * ny * nx;
    for (int k = 0; k < 13; k++) rec_i[k] = 0;
    for (int k = 0; k < 6; k++) rec_f[k] = NAN;
    rec_i[0] = ST_UNCERTAIN; rec_i[3] = n; rec_i[7] = -1;
    /* finiteness, zero boundary, sampling domain (certify_map :412-425; interpolation.py:43 check_map_domain) */
    for (int64_t i = 0; i < 3 * nn; i++) if (!fin(u[i])) { rec_i[1] = R_NONFINITE; return; }
    for (int64_t z = 0; z < nz; z++)
        for (int64_t y = 0; y < ny; y++)
            for (int64_t x = 0; x < nx; x++) {
                int face = z == 0 || z == nz - 1 || y == 0 || y == ny - 1 || x == 0 || x == nx - 1;
                if (!face) continue;
                const double *q = u + 3 * ((z * ny + y) * nx + x);
                if (q[0] != 0 || q[1] != 0 || q[2] != 0) { rec_i[0] = ST_INFEASIBLE; rec_i[1] = R_BOUNDARY; return; }
            }
    int64_t invalid = 0;
    for (int64_t z = 0; z < nz; z++)
        for (int64_t y = 0; y < ny; y++)
            for (int64_t x = 0; x < nx; x++) {
                const double *q = u + 3 * ((z * ny + y) * nx + x);
                int interior = z > 0 && z < nz - 1 && y > 0 && y < ny - 1 && x > 0 && x < nx - 1;
                const double *ax[3] = {axx, axy, axz};
                int64_t idx[3] = {x, y, z}, len[3] = {nx, ny, nz};
                int bad = 0;
                for (int j = 0; j < 3; j++) {
                    double value = q[j] + ax[j][idx[j]], lo = ax[j][0], hi = ax[j][len[j] - 1];
                    if (!fin(value) || value < lo || value > hi) bad = 1;
                    if (interior && (value <= lo || value >= hi)) bad = 1;
                }
                invalid += bad;
            }
    if (invalid) { rec_i[0] = ST_INFEASIBLE; rec_i[1] = R_DOMAIN; return; }

    double *margin = (double *)malloc(sizeof(double) * (size_t)n);
    uint8_t *flag = (uint8_t *)malloc((size_t)n);
    uint8_t *stage = (uint8_t *)calloc((size_t)n, 1);        /* 1 hull-proven, 2 prescreen-proven, 3 fallback */
    if (use_hull) {
        oc_edge_hull(u, nz, ny, nx, spacing, delta, 0, n, margin, flag);
    } else {                                 /* whole-cell Bernstein execution: no preproof (feasibility.py:447) */
        for (int64_t c = 0; c < n; c++) { margin[c] = NAN; flag[c] = 1; }
        use_prescreen = 0;
    }
    int64_t unknown = 0, bad = 0, boxes = 0, maxd = 0, fast = 0, fallback = 0, prescreened = 0;
    int64_t witness_cell = -1;
    double wpt[3] = {NAN, NAN, NAN};
    double lowest = INFINITY;
    int any_margin = 0, arith = 0;
    double sampled_min = INFINITY;
    for (int64_t t0 = 0; t0 < n; t0 += tile_size) {
        int64_t t1 = t0 + tile_size < n ? t0 + tile_size : n;
        int flagged = 0;
        for (int64_t c = t0; c < t1; c++) flagged |= flag[c];
        for (int64_t c = t0; c < t1; c++) {
            if (!flagged && margin[c] > 0) {
                stage[c] = 1; fast++; boxes++;
                if (margin[c] < lowest) lowest = margin[c];
                any_margin = 1;
            } else {
                stage[c] = 3; fallback++;
            }
        }
    }
    if (use_prescreen && fallback) {
        int64_t m = 0;
        int64_t *cells = (int64_t *)malloc(sizeof(int64_t) * (size_t)fallback);
        for (int64_t c = 0; c < n; c++) if (stage[c] == 3) cells[m++] = c;
        double *lower = (double *)malloc(sizeof(double) * (size_t)m);
        oc_prescreen(u, nz, ny, nx, D, cells, 0, m, g12, g6, g3, sq27, eta, lower);
        for (int64_t i = 0; i < m; i++) {
            double mp = delta == 0. ? lower[i] : nextafter(lower[i] - delta, -INFINITY);
            if (mp > 0) {
                stage[cells[i]] = 2; prescreened++; boxes++;
                if (mp < lowest) lowest = mp;
                any_margin = 1;
            }
        }
        fallback -= prescreened;
        free(lower); free(cells);
    }
    /* fallback jobs: one per tile, in tile order; a failed cell voids the whole job */
    double v[24], plo[27], phi[27], clo[27], chi[27], smp[27];
    for (int64_t t0 = 0; t0 < n; t0 += tile_size) {
        int64_t t1 = t0 + tile_size < n ? t0 + tile_size : n;
        int64_t count = 0;
        int job_ok = 1;
        for (int64_t c = t0; c < t1; c++) {
            if (stage[c] != 3) continue;
            count++;
            int64_t cx = nx - 1, cy = ny - 1;
            int64_t x0 = c % cx, y0 = (c / cx) % cy, z0 = c / (cx * cy), base = (z0 * ny + y0) * nx + x0;
            for (int a = 0; a < 8; a++)
                for (int r = 0; r < 3; r++) v[3 * a + r] = u[3 * vnode(base, a, ny, nx) + r];
            job_ok &= oc_fallback_cell(v, spacing, delta, plo, phi, clo, chi, smp);
        }
        if (!count) continue;
        if (!job_ok) { arith = 1; unknown += count; continue; }
        boxes += count;
        double safe_min = INFINITY;
        int any_safe = 0;
        for (int64_t c = t0; c < t1; c++) {
            if (stage[c] != 3) continue;
            int64_t cx = nx - 1, cy = ny - 1;
            int64_t x0 = c % cx, y0 = (c / cx) % cy, z0 = c / (cx * cy), base = (z0 * ny + y0) * nx + x0;
            for (int a = 0; a < 8; a++)
                for (int r = 0; r < 3; r++) v[3 * a + r] = u[3 * vnode(base, a, ny, nx) + r];
            oc_fallback_cell(v, spacing, delta, plo, phi, clo, chi, smp);
            for (int q = 0; q < 27; q++) if (smp[q] < sampled_min) sampled_min = smp[q];
            double mn = min27(clo);
            if (mn > 0) { any_safe = 1; if (mn < safe_min) safe_min = mn; continue; }
            cls_t r;
            oc_classify(clo, chi, plo, phi, delta, max_depth, max_boxes, depth_first, &r);
            if (r.has_margin) { if (r.margin < lowest) lowest = r.margin; any_margin = 1; }
            if (r.reason == R_ARITH) arith = 1;
            boxes += r.boxes - 1;
            if (r.depth > maxd) maxd = r.depth;
            unknown += r.status == ST_UNCERTAIN;
            bad += r.status == ST_INFEASIBLE;
            if (r.status == ST_INFEASIBLE && witness_cell < 0) {
                witness_cell = c;
                if (r.has_witness) { wpt[0] = r.witness[0]; wpt[1] = r.witness[1]; wpt[2] = r.witness[2]; }
            }
        }
        if (any_safe) { if (safe_min < lowest) lowest = safe_min; any_margin = 1; }
    }
    int status = bad ? ST_INFEASIBLE : (unknown ? ST_UNCERTAIN : ST_FEASIBLE);
    int reason = bad ? R_VIOLATION : (arith ? R_ARITH : (unknown ? R_SUBDIV_BUDGET : R_BERNSTEIN));
    if ((fast || prescreened) && status == ST_FEASIBLE) reason = R_ENCLOSURE;
    rec_i[0] = status; rec_i[1] = reason; rec_i[2] = n; rec_i[3] = unknown; rec_i[4] = bad; rec_i[5] = boxes;
    rec_i[6] = maxd; rec_i[7] = witness_cell; rec_i[8] = fast; rec_i[9] = fallback; rec_i[10] = prescreened;
    if (!use_hull) rec_i[9] = 0;   /* the plain FeasibilityResult has no stage counts */
    if (any_margin && !arith) {
        rec_f[1] = lowest;
        rec_f[0] = delta == 0. ? lowest : nextafter(lowest + delta, -INFINITY);
        rec_i[11] = 1;
    }
    if (!(fast || prescreened) && fin(sampled_min)) { rec_f[2] = sampled_min; rec_i[12] = 1; }
    rec_f[3] = wpt[0]; rec_f[4] = wpt[1]; rec_f[5] = wpt[2];
    free(margin); free(flag); free(stage);
}
