/*
 * ORACLE — test infrastructure, never product code.
 *
 * A plain-C restatement of the OWT-Krylov single-rank solve path, written
 * from the reference's documented behaviour.  Only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg load it, and only as the checker.  It is
 * pinned against the reference itself (oracle/_ref, built by oracle/Makefile
 * from the unmodified reference headers) and against the known-answer values
 * of the reference's own unit tests (tests/golden/).
 *
 * Arithmetic follows the reference as it ships (-O3, no -march, so no FMA
 * contraction); this file is compiled with -ffp-contract=off for the same
 * reason.  Indices are int64 (the reference uses size_t).
 *
 * Reference file:line anchors are into include/owt/krylov/ of the reference.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef int64_t i64;

enum { ORC_OK = 0, ORC_INVALID = 1, ORC_ZERO_PIVOT = 2, ORC_RANGE = 3 };

/* ------------------------------------------------------------------ SpMV */

/* block_csr.hpp:198-215 — y[r,c] = sum_e val[e,c] * x[col[e],c], entry order. */
void orc_bsr_spmv(i64 owned, i64 bs, const i64* rp, const i64* ci,
                  const double* v, const double* x, double* y)
{
    for (i64 r = 0; r < owned; ++r) {
        double* out = y + r * bs;
        for (i64 c = 0; c < bs; ++c) out[c] = 0.0;
        for (i64 e = rp[r]; e < rp[r + 1]; ++e) {
            const double* in = x + ci[e] * bs;
            const double* a = v + e * bs;
            for (i64 c = 0; c < bs; ++c) out[c] += a[c] * in[c];
        }
    }
}

/* split_block_csr.hpp:95-119 — y = diag*x + sum_e off[e]*x[col]. */
void orc_split_spmv(i64 owned, i64 bs, const i64* rp, const i64* ci,
                    const double* diag, const double* off, const double* x, double* y)
{
    for (i64 r = 0; r < owned; ++r) {
        double* out = y + r * bs;
        for (i64 c = 0; c < bs; ++c) out[c] = diag[r * bs + c] * x[r * bs + c];
        for (i64 e = rp[r]; e < rp[r + 1]; ++e) {
            const double* in = x + ci[e] * bs;
            const double* a = off + e * bs;
            for (i64 c = 0; c < bs; ++c) out[c] += a[c] * in[c];
        }
    }
}

/* dense_block_csr.hpp:179-205 — per entry, a block-row dot, then accumulate. */
void orc_dense_spmv(i64 owned, i64 bs, const i64* rp, const i64* ci,
                    const double* v, const double* x, double* y)
{
    for (i64 r = 0; r < owned; ++r) {
        double* out = y + r * bs;
        for (i64 c = 0; c < bs; ++c) out[c] = 0.0;
        for (i64 e = rp[r]; e < rp[r + 1]; ++e) {
            const double* in = x + ci[e] * bs;
            const double* b = v + e * bs * bs;
            for (i64 br = 0; br < bs; ++br) {
                double contribution = 0.0;
                for (i64 bc = 0; bc < bs; ++bc) contribution += b[br * bs + bc] * in[bc];
                out[br] += contribution;
            }
        }
    }
}

/* ------------------------------------------------------------ reductions */

/* reduction.hpp:114-145 — eight strided partial sums, then a fixed tree. */
double orc_dot(i64 n, const double* a, const double* b)
{
    double p[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    i64 i = 0;
    for (; i + 8 <= n; i += 8)
        for (int l = 0; l < 8; ++l) p[l] += a[i + l] * b[i + l];
    double s = (p[0] + p[1]) + (p[2] + p[3]) + (p[4] + p[5]) + (p[6] + p[7]);
    for (; i < n; ++i) s += a[i] * b[i];
    return s;
}

/* reduction.hpp:64-89 — max-scaled, Neumaier-compensated two-pass norm. */
double orc_norm(i64 n, const double* a)
{
    double scale = 0.0;
    for (i64 i = 0; i < n; ++i) {
        const double m = fabs(a[i]);
        if (isnan(m)) return NAN;
        if (m > scale) scale = m;
    }
    if (scale == 0.0 || isinf(scale)) return scale;
    double sum = 0.0, corr = 0.0;
    for (i64 i = 0; i < n; ++i) {
        const double ratio = a[i] / scale;
        const double term = ratio * ratio;
        const double upd = sum + term;
        corr += sum >= term ? (sum - upd) + term : (term - upd) + sum;
        sum = upd;
    }
    return scale * sqrt(sum + corr);
}

/* ------------------------------------------------------- preconditioners */

/* block_csr.hpp:217-236 — first entry with column == row is the diagonal. */
static int bsr_diagonal(i64 owned, i64 bs, const i64* rp, const i64* ci,
                        const double* v, double* d)
{
    for (i64 r = 0; r < owned; ++r) {
        int found = 0;
        for (i64 e = rp[r]; e < rp[r + 1]; ++e) {
            if (ci[e] == r) {
                memcpy(d + r * bs, v + e * bs, (size_t)bs * sizeof(double));
                found = 1;
                break;
            }
        }
        if (!found) return ORC_INVALID;
    }
    return ORC_OK;
}

/* preconditioner.hpp:55-71 — reciprocal diagonal, singular-diagonal check. */
int orc_jacobi_inverse(i64 owned, i64 bs, const i64* rp, const i64* ci,
                       const double* v, const double* split_diag,
                       double minimum_diagonal, double* inv)
{
    const i64 n = owned * bs;
    if (split_diag) memcpy(inv, split_diag, (size_t)n * sizeof(double));
    else if (bsr_diagonal(owned, bs, rp, ci, v, inv) != ORC_OK) return ORC_INVALID;
    for (i64 i = 0; i < n; ++i) {
        const double d = inv[i];
        if (!isfinite(d) || fabs(d) <= minimum_diagonal) return ORC_INVALID;
        inv[i] = 1.0 / d;
    }
    return ORC_OK;
}

/* preconditioner.hpp:78-85 */
void orc_jacobi_apply(i64 n, const double* inv, const double* in, double* out)
{
    for (i64 i = 0; i < n; ++i) out[i] = inv[i] * in[i];
}

/* preconditioner.hpp:142-174 (diagonal cache) and :181-239 (apply):
 * forward (D + wL) sweep into work, zero output, backward sweep, scale w(2-w). */
int orc_ssor_apply(i64 owned, i64 bs, const i64* rp, const i64* ci,
                   const double* v, double omega, const double* in, double* out,
                   double* work)
{
    double* d = (double*)malloc((size_t)(owned * bs) * sizeof(double));
    if (bsr_diagonal(owned, bs, rp, ci, v, d) != ORC_OK) { free(d); return ORC_INVALID; }
    for (i64 r = 0; r < owned; ++r) {
        double* y = work + r * bs;
        memcpy(y, in + r * bs, (size_t)bs * sizeof(double));
        for (i64 e = rp[r]; e < rp[r + 1]; ++e) {
            const i64 col = ci[e];
            if (col >= r || col >= owned) continue;
            for (i64 c = 0; c < bs; ++c) y[c] -= omega * v[e * bs + c] * work[col * bs + c];
        }
        for (i64 c = 0; c < bs; ++c) y[c] /= d[r * bs + c];
    }
    for (i64 i = 0; i < owned * bs; ++i) out[i] = 0.0;
    for (i64 r = owned - 1; r >= 0; --r) {
        double* z = out + r * bs;
        const double* y = work + r * bs;
        for (i64 c = 0; c < bs; ++c) z[c] = d[r * bs + c] * y[c];
        for (i64 e = rp[r]; e < rp[r + 1]; ++e) {
            const i64 col = ci[e];
            if (col <= r || col >= owned) continue;
            for (i64 c = 0; c < bs; ++c) z[c] -= omega * v[e * bs + c] * out[col * bs + c];
        }
        for (i64 c = 0; c < bs; ++c) z[c] /= d[r * bs + c];
    }
    const double s = omega * (2.0 - omega);
    for (i64 i = 0; i < owned * bs; ++i) out[i] *= s;
    free(d);
    return ORC_OK;
}

/* split_block_csr.hpp:243-309 — same sweeps on the split layout; no output
 * clear, and the final scale only when omega != 1. */
void orc_split_ssor_apply(i64 owned, i64 bs, const i64* rp, const i64* ci,
                          const double* diag, const double* off, double omega,
                          const double* in, double* out, double* work)
{
    for (i64 r = 0; r < owned; ++r) {
        double* f = work + r * bs;
        memcpy(f, in + r * bs, (size_t)bs * sizeof(double));
        for (i64 e = rp[r]; e < rp[r + 1]; ++e) {
            const i64 col = ci[e];
            if (col >= r || col >= owned) continue;
            for (i64 c = 0; c < bs; ++c) f[c] -= omega * off[e * bs + c] * work[col * bs + c];
        }
        for (i64 c = 0; c < bs; ++c) f[c] /= diag[r * bs + c];
    }
    for (i64 r = owned - 1; r >= 0; --r) {
        double* z = out + r * bs;
        const double* f = work + r * bs;
        for (i64 c = 0; c < bs; ++c) z[c] = diag[r * bs + c] * f[c];
        for (i64 e = rp[r]; e < rp[r + 1]; ++e) {
            const i64 col = ci[e];
            if (col <= r || col >= owned) continue;
            for (i64 c = 0; c < bs; ++c) z[c] -= omega * off[e * bs + c] * out[col * bs + c];
        }
        for (i64 c = 0; c < bs; ++c) z[c] /= diag[r * bs + c];
    }
    if (omega != 1.0) {
        const double s = omega * (2.0 - omega);
        for (i64 i = 0; i < owned * bs; ++i) out[i] *= s;
    }
}

/* ----------------------------------------------------------------- ILU(k) */

typedef struct {
    i64 owned, bs, fill_level, entries, capacity;
    i64* rp;        /* owned+1 */
    i64* ci;        /* entries, sorted per row */
    i64* lev;       /* symbolic fill level per entry */
    i64* src;       /* source entry in the matrix, or -1 for fill */
    i64* diagpos;   /* owned */
    i64* counts;    /* local entries per matrix row */
    double* val;    /* entries * bs */
    double* inv;    /* owned * bs */
} orc_ilu;

static void ilu_push(orc_ilu* h, i64 col, i64 lev, i64 src)
{
    if (h->entries == h->capacity) {
        h->capacity = h->capacity ? 2 * h->capacity : 1024;
        h->ci = (i64*)realloc(h->ci, (size_t)h->capacity * sizeof(i64));
        h->lev = (i64*)realloc(h->lev, (size_t)h->capacity * sizeof(i64));
        h->src = (i64*)realloc(h->src, (size_t)h->capacity * sizeof(i64));
    }
    h->ci[h->entries] = col;
    h->lev[h->entries] = lev;
    h->src[h->entries] = src;
    h->entries++;
}

/* Row scratch: a column-sorted array of (column, level, source). */
typedef struct { i64 col, lev, src; } row_entry;

static int row_insert(row_entry* row, i64* len, i64 col, i64 lev, i64 src, int unique)
{
    i64 lo = 0, hi = *len;
    while (lo < hi) {
        const i64 mid = (lo + hi) / 2;
        if (row[mid].col < col) lo = mid + 1; else hi = mid;
    }
    if (lo < *len && row[lo].col == col) {
        if (unique) return -1;
        if (lev < row[lo].lev) row[lo].lev = lev;
        return 0;
    }
    memmove(row + lo + 1, row + lo, (size_t)(*len - lo) * sizeof(row_entry));
    row[lo].col = col; row[lo].lev = lev; row[lo].src = src;
    ++*len;
    return 1;
}

static int ilu_factorize(orc_ilu* h);

/* preconditioner.hpp:373-427 — symbolic ILU(k): ghost columns dropped, sorted
 * columns, level(i,j) = min(level(i,p) + level(p,j) + 1), fill kept while the
 * level stays <= k; a duplicate column or a missing diagonal is rejected. */
orc_ilu* orc_ilu_create(i64 owned, i64 bs, const i64* rp, const i64* ci,
                        const double* v, i64 fill_level, int* status)
{
    orc_ilu* h = (orc_ilu*)calloc(1, sizeof(orc_ilu));
    h->owned = owned; h->bs = bs; h->fill_level = fill_level;
    h->rp = (i64*)calloc((size_t)owned + 1, sizeof(i64));
    h->diagpos = (i64*)calloc((size_t)owned, sizeof(i64));
    h->counts = (i64*)calloc((size_t)owned, sizeof(i64));
    i64 cap = 64;
    row_entry* row = (row_entry*)malloc((size_t)cap * sizeof(row_entry));
    *status = ORC_OK;
    for (i64 r = 0; r < owned && *status == ORC_OK; ++r) {
        i64 len = 0;
        for (i64 s = rp[r]; s < rp[r + 1]; ++s) {
            if (ci[s] >= owned) continue;
            if (len + 1 > cap) { cap *= 2; row = (row_entry*)realloc(row, (size_t)cap * sizeof(row_entry)); }
            if (row_insert(row, &len, ci[s], 0, s, 1) < 0) { *status = ORC_INVALID; break; }
            h->counts[r]++;
        }
        if (*status != ORC_OK) break;
        /* Pivots are visited in column order; fill inserted to the right of the
         * current pivot is visited later, as std::map iteration does. */
        for (i64 k = 0; k < len && row[k].col < r; ++k) {
            const i64 pivot = row[k].col, lower = row[k].lev;
            if (lower >= fill_level) continue;
            for (i64 u = h->diagpos[pivot] + 1; u < h->rp[pivot + 1]; ++u) {
                if (h->lev[u] > fill_level - lower - 1) continue;
                if (len + 1 > cap) { cap *= 2; row = (row_entry*)realloc(row, (size_t)cap * sizeof(row_entry)); }
                row_insert(row, &len, h->ci[u], lower + h->lev[u] + 1, -1, 0);
            }
        }
        int found = 0;
        for (i64 k = 0; k < len; ++k) {
            if (row[k].col == r) { h->diagpos[r] = h->entries; found = 1; }
            ilu_push(h, row[k].col, row[k].lev, row[k].src);
        }
        if (!found) { *status = ORC_INVALID; break; }
        h->rp[r + 1] = h->entries;
    }
    free(row);
    if (*status != ORC_OK) return h;
    h->val = (double*)calloc((size_t)(h->entries * bs) + 1, sizeof(double));
    h->inv = (double*)calloc((size_t)(owned * bs), sizeof(double));
    for (i64 e = 0; e < h->entries; ++e)
        if (h->src[e] >= 0) memcpy(h->val + e * bs, v + h->src[e] * bs, (size_t)bs * sizeof(double));
    *status = ilu_factorize(h);
    return h;
}

/* preconditioner.hpp:429-437 — linear search for a column in a factor row. */
static i64 ilu_find(const orc_ilu* h, i64 r, i64 col)
{
    for (i64 e = h->rp[r]; e < h->rp[r + 1]; ++e)
        if (h->ci[e] == col) return e;
    return -1;
}

/* preconditioner.hpp:439-485 — component-wise IKJ elimination, pivot
 * tolerance 64*eps, stored reciprocal diagonal. */
static int ilu_factorize(orc_ilu* h)
{
    const double tol = 64.0 * DBL_EPSILON;
    const i64 bs = h->bs;
    for (i64 r = 0; r < h->owned; ++r) {
        for (i64 l = h->rp[r]; l < h->diagpos[r]; ++l) {
            const i64 p = h->ci[l];
            double* lv = h->val + l * bs;
            const double* piv = h->val + h->diagpos[p] * bs;
            for (i64 c = 0; c < bs; ++c) {
                if (fabs(piv[c]) <= tol) return ORC_ZERO_PIVOT;
                lv[c] /= piv[c];
            }
            for (i64 u = h->diagpos[p] + 1; u < h->rp[p + 1]; ++u) {
                const i64 t = ilu_find(h, r, h->ci[u]);
                if (t < 0) continue;
                double* tv = h->val + t * bs;
                const double* uv = h->val + u * bs;
                for (i64 c = 0; c < bs; ++c) tv[c] -= lv[c] * uv[c];
            }
        }
    }
    for (i64 r = 0; r < h->owned; ++r) {
        const double* d = h->val + h->diagpos[r] * bs;
        for (i64 c = 0; c < bs; ++c) {
            if (!isfinite(d[c]) || fabs(d[c]) <= tol) return ORC_ZERO_PIVOT;
            h->inv[r * bs + c] = 1.0 / d[c];
        }
    }
    return ORC_OK;
}

/* preconditioner.hpp:269-311 — same pattern required; copy values, refactor. */
int orc_ilu_update(orc_ilu* h, const i64* rp, const i64* ci, const double* v)
{
    const i64 bs = h->bs;
    for (i64 r = 0; r < h->owned; ++r) {
        i64 count = 0;
        for (i64 s = rp[r]; s < rp[r + 1]; ++s) count += ci[s] < h->owned;
        if (count != h->counts[r]) return ORC_INVALID;
        for (i64 e = h->rp[r]; e < h->rp[r + 1]; ++e) {
            const i64 s = h->src[e];
            if (s < 0) { memset(h->val + e * bs, 0, (size_t)bs * sizeof(double)); continue; }
            if (s < rp[r] || s >= rp[r + 1] || ci[s] != h->ci[e]) return ORC_INVALID;
            memcpy(h->val + e * bs, v + s * bs, (size_t)bs * sizeof(double));
        }
    }
    return ilu_factorize(h);
}

/* preconditioner.hpp:320-363 — unit-L forward solve into out, then backward
 * U solve with the reciprocal diagonal; in == out is allowed. */
void orc_ilu_apply(const orc_ilu* h, const double* in, double* out)
{
    const i64 bs = h->bs;
    for (i64 r = 0; r < h->owned; ++r) {
        double* y = out + r * bs;
        if (in != out) memcpy(y, in + r * bs, (size_t)bs * sizeof(double));
        for (i64 e = h->rp[r]; e < h->diagpos[r]; ++e) {
            const double* f = h->val + e * bs;
            const double* prev = out + h->ci[e] * bs;
            for (i64 c = 0; c < bs; ++c) y[c] -= f[c] * prev[c];
        }
    }
    for (i64 r = h->owned - 1; r >= 0; --r) {
        double* x = out + r * bs;
        for (i64 e = h->diagpos[r] + 1; e < h->rp[r + 1]; ++e) {
            const double* f = h->val + e * bs;
            const double* prev = out + h->ci[e] * bs;
            for (i64 c = 0; c < bs; ++c) x[c] -= f[c] * prev[c];
        }
        for (i64 c = 0; c < bs; ++c) x[c] *= h->inv[r * bs + c];
    }
}

i64 orc_ilu_entries(const orc_ilu* h) { return h->entries; }

void orc_ilu_copy(const orc_ilu* h, i64* rp, i64* ci, double* val, double* inv,
                  i64* diagpos, i64* src)
{
    if (rp) memcpy(rp, h->rp, (size_t)(h->owned + 1) * sizeof(i64));
    if (ci) memcpy(ci, h->ci, (size_t)h->entries * sizeof(i64));
    if (val) memcpy(val, h->val, (size_t)(h->entries * h->bs) * sizeof(double));
    if (inv) memcpy(inv, h->inv, (size_t)(h->owned * h->bs) * sizeof(double));
    if (diagpos) memcpy(diagpos, h->diagpos, (size_t)h->owned * sizeof(i64));
    if (src) memcpy(src, h->src, (size_t)h->entries * sizeof(i64));
}

void orc_ilu_destroy(orc_ilu* h)
{
    if (!h) return;
    free(h->rp); free(h->ci); free(h->lev); free(h->src); free(h->diagpos);
    free(h->counts); free(h->val); free(h->inv); free(h);
}

/* ------------------------------------------------------------ level sets */

/* Level sets have no counterpart in the reference (it sweeps rows in order).
 * Definition used by the device sweeps: a row's lower level is 0 without a
 * local dependency below it, else 1 + the maximum lower level of its columns
 * c < row; the upper level mirrors it for columns row < c < owned, computed
 * from the last row upward.  Ghost columns (>= owned) are not dependencies. */
void orc_levels(i64 owned, const i64* rp, const i64* ci, i64* lower, i64* upper)
{
    for (i64 r = 0; r < owned; ++r) {
        i64 lv = 0;
        for (i64 e = rp[r]; e < rp[r + 1]; ++e) {
            const i64 c = ci[e];
            if (c < r && lower[c] + 1 > lv) lv = lower[c] + 1;
        }
        lower[r] = lv;
    }
    for (i64 r = owned - 1; r >= 0; --r) {
        i64 lv = 0;
        for (i64 e = rp[r]; e < rp[r + 1]; ++e) {
            const i64 c = ci[e];
            if (c > r && c < owned && upper[c] + 1 > lv) lv = upper[c] + 1;
        }
        upper[r] = lv;
    }
}

/* -------------------------------------------------------------- orderings */

/* ordering.hpp:31-49 + :138-180 — reverse Cuthill-McKee.  Neighbours are
 * ordered by degree with an insertion sort: for lists of at most 16 elements
 * this is exactly what the reference's std::sort does (libstdc++ finishes
 * short ranges with a stable insertion sort), which covers triangle meshes. */
int orc_rcm(i64 owned, const i64* rp, const i64* ci, i64* out)
{
    i64* grp = (i64*)calloc((size_t)owned + 1, sizeof(i64));
    i64* deg = (i64*)calloc((size_t)owned, sizeof(i64));
    i64 total = rp[owned];
    i64* g = (i64*)malloc((size_t)(total > 0 ? total : 1) * sizeof(i64));
    i64 k = 0;
    for (i64 r = 0; r < owned; ++r) {
        const i64 start = k;
        for (i64 e = rp[r]; e < rp[r + 1]; ++e) {
            const i64 c = ci[e];
            if (c < owned && c != r) g[k++] = c;
        }
        /* sort + unique the adjacency list */
        for (i64 a = start + 1; a < k; ++a) {
            const i64 t = g[a];
            i64 b = a;
            while (b > start && g[b - 1] > t) { g[b] = g[b - 1]; --b; }
            g[b] = t;
        }
        i64 w = start;
        for (i64 a = start; a < k; ++a)
            if (a == start || g[a] != g[a - 1]) g[w++] = g[a];
        k = w;
        grp[r + 1] = k;
        deg[r] = k - start;
    }
    char* visited = (char*)calloc((size_t)owned, 1);
    i64* queue = (i64*)malloc((size_t)owned * sizeof(i64));
    i64* nb = (i64*)malloc((size_t)(owned > 0 ? owned : 1) * sizeof(i64));
    i64 count = 0;
    while (count < owned) {
        i64 seed = owned;
        for (i64 v = 0; v < owned; ++v)
            if (!visited[v] && (seed == owned || deg[v] < deg[seed])) seed = v;
        i64 head = 0, tail = 0;
        queue[tail++] = seed;
        visited[seed] = 1;
        while (head < tail) {
            const i64 v = queue[head++];
            out[count++] = v;
            i64 m = 0;
            for (i64 e = grp[v]; e < grp[v + 1]; ++e)
                if (!visited[g[e]]) nb[m++] = g[e];
            for (i64 a = 1; a < m; ++a) {
                const i64 t = nb[a];
                i64 b = a;
                while (b > 0 && deg[nb[b - 1]] > deg[t]) { nb[b] = nb[b - 1]; --b; }
                nb[b] = t;
            }
            for (i64 a = 0; a < m; ++a)
                if (!visited[nb[a]]) { visited[nb[a]] = 1; queue[tail++] = nb[a]; }
        }
    }
    for (i64 a = 0, b = owned - 1; a < b; ++a, --b) { const i64 t = out[a]; out[a] = out[b]; out[b] = t; }
    free(grp); free(deg); free(g); free(visited); free(queue); free(nb);
    return ORC_OK;
}

/* ordering.hpp:51-77 — Hilbert index on a power-of-two grid. */
static uint64_t hilbert_index(uint32_t x, uint32_t y, uint32_t extent)
{
    uint64_t index = 0;
    for (uint32_t s = extent / 2; s > 0; s /= 2) {
        const uint32_t rx = (x & s) != 0, ry = (y & s) != 0;
        index += (uint64_t)s * s * ((3u * rx) ^ ry);
        if (ry == 0) {
            if (rx == 1) { x = s - 1 - x; y = s - 1 - y; }
            const uint32_t t = x; x = y; y = t;
        }
    }
    return index;
}

typedef struct { uint64_t key; i64 node; } keyed;
static int keyed_cmp(const void* a, const void* b)
{
    const keyed* p = (const keyed*)a; const keyed* q = (const keyed*)b;
    if (p->key != q->key) return p->key < q->key ? -1 : 1;
    return p->node < q->node ? -1 : (p->node > q->node);
}

/* ordering.hpp:231-261 — 2^16 grid on bounding-box-normalised coordinates,
 * sorted by (index, node). */
int orc_hilbert(i64 n, const double* xy, i64* out)
{
    if (n == 0) return ORC_OK;
    double x0 = xy[0], x1 = xy[0], y0 = xy[1], y1 = xy[1];
    for (i64 i = 0; i < n; ++i) {
        const double x = xy[2 * i], y = xy[2 * i + 1];
        if (x < x0) x0 = x; if (x > x1) x1 = x;
        if (y < y0) y0 = y; if (y > y1) y1 = y;
    }
    const uint32_t extent = 1u << 16;
    keyed* k = (keyed*)malloc((size_t)n * sizeof(keyed));
    const double wx = (x1 - x0) > DBL_EPSILON ? (x1 - x0) : DBL_EPSILON;
    const double wy = (y1 - y0) > DBL_EPSILON ? (y1 - y0) : DBL_EPSILON;
    for (i64 i = 0; i < n; ++i) {
        double nx = (xy[2 * i] - x0) / wx, ny = (xy[2 * i + 1] - y0) / wy;
        nx = nx < 0.0 ? 0.0 : (nx > 1.0 ? 1.0 : nx);
        ny = ny < 0.0 ? 0.0 : (ny > 1.0 ? 1.0 : ny);
        k[i].key = hilbert_index((uint32_t)(nx * (extent - 1)), (uint32_t)(ny * (extent - 1)), extent);
        k[i].node = i;
    }
    qsort(k, (size_t)n, sizeof(keyed), keyed_cmp);
    for (i64 i = 0; i < n; ++i) out[i] = k[i].node;
    free(k);
    return ORC_OK;
}

/* ---------------------------------------------------------------- solvers */

typedef struct {
    double relative_tolerance, absolute_tolerance, breakdown_tolerance;
    uint64_t maximum_iterations, convergence_check_interval, restart;
    uint64_t residual_replacement_interval, idr_shadow_space;
    double relaxation;
    int32_t verify_true_residual, gmres_orthogonalization;
} orc_options;

typedef struct {
    int32_t status, breakdown_reason;
    uint64_t iterations, operator_applications, preconditioner_applications;
    uint64_t global_reductions, reorthogonalizations, arnoldi_norm_verifications;
    double initial_residual_norm, recursive_residual_norm, true_residual_norm, relative_residual_norm;
    int32_t converged_by_application, pad;
    double solve_seconds;
} orc_result;

/* core.hpp:24-30 and :41-52 */
enum { ST_CONVERGED, ST_MAXIT, ST_BREAKDOWN, ST_DIVERGED, ST_INVALID };
enum { BR_NONE, BR_ARNOLDI, BR_SINGULAR, BR_BIORTH, BR_ALPHA, BR_OMEGA_DEN, BR_OMEGA_ZERO,
       BR_IDR_SHADOW, BR_IDR_SMALL, BR_NONFINITE };

/* Operator (matrix kinds: 0 BSR, 1 split, 2 dense) and preconditioner
 * (0 identity, 1 Jacobi, 2 SSOR, 3 split SSOR, 4 ILU). */
typedef struct {
    int kind;
    i64 owned, ghost, bs;
    const i64* rp; const i64* ci; const double* v; const double* diag; const double* off;
} orc_matrix;

typedef struct {
    int kind;
    double omega;
    const double* inv;   /* Jacobi */
    const orc_ilu* ilu;  /* ILU */
    double* work;        /* SSOR scratch, owned*bs */
} orc_pc;

static void op_apply(const orc_matrix* m, const double* x, double* y, orc_result* res)
{
    if (m->kind == 0) orc_bsr_spmv(m->owned, m->bs, m->rp, m->ci, m->v, x, y);
    else if (m->kind == 1) orc_split_spmv(m->owned, m->bs, m->rp, m->ci, m->diag, m->off, x, y);
    else orc_dense_spmv(m->owned, m->bs, m->rp, m->ci, m->v, x, y);
    res->operator_applications++;
}

static void pc_apply(const orc_matrix* m, const orc_pc* p, const double* in, double* out, orc_result* res)
{
    const i64 n = m->owned * m->bs;
    switch (p->kind) {
    case 0: if (in != out) memcpy(out, in, (size_t)n * sizeof(double)); break;
    case 1: orc_jacobi_apply(n, p->inv, in, out); break;
    case 2: orc_ssor_apply(m->owned, m->bs, m->rp, m->ci, m->v, p->omega, in, out, p->work); break;
    case 3: orc_split_ssor_apply(m->owned, m->bs, m->rp, m->ci, m->diag, m->off, p->omega, in, out, p->work); break;
    default: orc_ilu_apply(p->ilu, in, out); break;
    }
    res->preconditioner_applications++;
}

static int valid_options(const orc_options* o)
{
    return isfinite(o->relative_tolerance) && isfinite(o->absolute_tolerance)
        && isfinite(o->breakdown_tolerance) && o->relative_tolerance >= 0
        && o->absolute_tolerance >= 0 && o->breakdown_tolerance > 0
        && o->maximum_iterations > 0 && o->convergence_check_interval > 0;
}

/* core.hpp:550-560 (without an application convergence test) */
static double threshold_of(double rhs_norm, const orc_options* o)
{
    const double rel = o->relative_tolerance * (rhs_norm > 0 ? rhs_norm : 1.0);
    if (!isfinite(rhs_norm) || !isfinite(rel)) return NAN;
    return o->absolute_tolerance > rel ? o->absolute_tolerance : rel;
}

static void init_result(orc_result* r)
{
    memset(r, 0, sizeof(*r));
    r->status = ST_INVALID;
    r->initial_residual_norm = r->recursive_residual_norm = NAN;
    r->true_residual_norm = r->relative_residual_norm = NAN;
}

static void set_residuals(orc_result* r, double rec, double tru, double rhs_norm)
{
    r->recursive_residual_norm = rec;
    r->true_residual_norm = tru;
    r->relative_residual_norm = tru / (rhs_norm > 0 ? rhs_norm : 1.0);
}

static double norm_r(i64 n, const double* a, orc_result* r) { r->global_reductions++; return orc_norm(n, a); }
static double dot_r(i64 n, const double* a, const double* b, orc_result* r) { r->global_reductions++; return orc_dot(n, a, b); }

/* krylov_solvers.hpp:62-74 */
static void true_residual(const orc_matrix* m, const double* b, const double* x, double* r,
                          double* work, orc_result* res)
{
    op_apply(m, x, work, res);
    for (i64 i = 0; i < m->owned * m->bs; ++i) r[i] = b[i] - work[i];
}

static void breakdown(orc_result* r, int reason) { r->status = ST_BREAKDOWN; r->breakdown_reason = reason; }

/* krylov_solvers.hpp:546-745 — preconditioned BiCGSTAB with typed breakdown
 * guards, false-convergence restart and periodic residual replacement.
 * Vectors must have room for ghosts: x and b are (owned+ghost)*bs. */
void orc_bicgstab(const orc_matrix* m, const orc_pc* p, const orc_options* o,
                  const double* b, double* x, orc_result* res)
{
    init_result(res);
    if (!valid_options(o)) return;
    const i64 n = m->owned * m->bs, nl = (m->owned + m->ghost) * m->bs;
    double* mem = (double*)calloc((size_t)(9 * nl), sizeof(double));
    double *r = mem, *sh = mem + nl, *ps = mem + 2 * nl, *pp = mem + 3 * nl, *v = mem + 4 * nl;
    double *s = mem + 5 * nl, *ss = mem + 6 * nl, *t = mem + 7 * nl, *w = mem + 8 * nl;
    true_residual(m, b, x, r, w, res);
    memcpy(sh, r, (size_t)n * sizeof(double));
    const double bnorm = norm_r(n, b, res), r0 = norm_r(n, r, res);
    const double thr = threshold_of(bnorm, o);
    const double tiny = 1024.0 * DBL_MIN;
    res->initial_residual_norm = r0;
    set_residuals(res, r0, r0, bnorm);
    if (!isfinite(r0) || !isfinite(thr)) { breakdown(res, BR_NONFINITE); goto done; }
    if (r0 <= thr) { res->status = ST_CONVERGED; goto done; }
    double rho_prev = 1, alpha = 1, omega = 1;
    int first = 1;
    for (uint64_t it = 1; it <= o->maximum_iterations; ++it) {
        res->iterations = it;
        const double rho = dot_r(n, sh, r, res);
        if (!isfinite(rho) || fabs(rho) <= tiny) { breakdown(res, isfinite(rho) ? BR_BIORTH : BR_NONFINITE); goto done; }
        if (first) { memcpy(ps, r, (size_t)n * sizeof(double)); first = 0; }
        else {
            if (fabs(omega) <= tiny) { breakdown(res, BR_OMEGA_ZERO); goto done; }
            const double beta = (rho / rho_prev) * (alpha / omega);
            for (i64 i = 0; i < n; ++i) ps[i] = r[i] + beta * (ps[i] - omega * v[i]);
        }
        pc_apply(m, p, ps, pp, res);
        op_apply(m, pp, v, res);
        const double sv = dot_r(n, sh, v, res);
        if (!isfinite(sv) || fabs(sv) <= tiny) { breakdown(res, isfinite(sv) ? BR_ALPHA : BR_NONFINITE); goto done; }
        alpha = rho / sv;
        for (i64 i = 0; i < n; ++i) s[i] = r[i] - alpha * v[i];
        const double snorm = norm_r(n, s, res);
        if (snorm <= thr) {
            for (i64 i = 0; i < n; ++i) x[i] += alpha * pp[i];
            true_residual(m, b, x, r, w, res);
            const double tn = norm_r(n, r, res);
            set_residuals(res, snorm, tn, bnorm);
            if (tn <= thr) { res->status = ST_CONVERGED; goto done; }
            memcpy(sh, r, (size_t)n * sizeof(double));
            memset(ps, 0, (size_t)n * sizeof(double));
            memset(v, 0, (size_t)n * sizeof(double));
            rho_prev = 1; alpha = 1; omega = 1; first = 1;
            continue;
        }
        pc_apply(m, p, s, ss, res);
        op_apply(m, ss, t, res);
        const double num = dot_r(n, t, s, res);
        const double den = dot_r(n, t, t, res);
        if (!isfinite(den) || fabs(den) <= tiny) { breakdown(res, isfinite(den) ? BR_OMEGA_DEN : BR_NONFINITE); goto done; }
        omega = num / den;
        const double angle = fabs(num) / sqrt(den) / snorm;
        if (!isfinite(omega) || omega == 0.0 || angle <= o->breakdown_tolerance) {
            breakdown(res, isfinite(omega) ? BR_OMEGA_ZERO : BR_NONFINITE); goto done;
        }
        for (i64 i = 0; i < n; ++i) x[i] += alpha * pp[i];
        for (i64 i = 0; i < n; ++i) x[i] += omega * ss[i];
        for (i64 i = 0; i < n; ++i) r[i] = s[i] - omega * t[i];
        const int replace = o->residual_replacement_interval > 0 && it % o->residual_replacement_interval == 0;
        const int check = it % o->convergence_check_interval == 0;
        if (replace || check) {
            const double rn = norm_r(n, r, res);
            if (replace || rn <= thr) {
                true_residual(m, b, x, r, w, res);
                const double tn = norm_r(n, r, res);
                set_residuals(res, rn, tn, bnorm);
                if (tn <= thr) { res->status = ST_CONVERGED; goto done; }
                memcpy(sh, r, (size_t)n * sizeof(double));
                memset(ps, 0, (size_t)n * sizeof(double));
                memset(v, 0, (size_t)n * sizeof(double));
                rho_prev = 1; alpha = 1; omega = 1; first = 1;
                continue;
            }
            res->recursive_residual_norm = rn;
        }
        rho_prev = rho;
    }
    {
        true_residual(m, b, x, r, w, res);
        const double tn = norm_r(n, r, res);
        set_residuals(res, res->recursive_residual_norm, tn, bnorm);
        res->status = tn <= thr ? ST_CONVERGED : ST_MAXIT;
        if (!isfinite(tn)) breakdown(res, BR_NONFINITE);
    }
done:
    free(mem);
}

/* krylov_solvers.hpp:24-40 — Neumaier-compensated correction sum. */
static void gmres_update(i64 n, const double* base, double* const* dirs, const double* coef,
                         i64 k, double* out)
{
    for (i64 i = 0; i < n; ++i) {
        double sum = 0, comp = 0;
        for (i64 j = 0; j < k; ++j) {
            const double term = coef[j] * dirs[j][i];
            const double upd = sum + term;
            comp += fabs(sum) >= fabs(term) ? (sum - upd) + term : (term - upd) + sum;
            sum = upd;
        }
        out[i] = base[i] + (sum + comp);
    }
}

/* krylov_solvers.hpp:159-486 — restarted right-preconditioned (F)GMRES with
 * iterated / adaptive / one-synchronisation classical Gram-Schmidt, norm
 * verification after cancellation, Givens rotations and a checked restart. */
void orc_gmres(const orc_matrix* m, const orc_pc* p, const orc_options* o,
               const double* b, double* x, orc_result* res)
{
    init_result(res);
    if (!valid_options(o) || o->restart == 0) return;
    const i64 n = m->owned * m->bs, nl = (m->owned + m->ghost) * m->bs;
    const i64 R = (i64)o->restart;
    double* mem = (double*)calloc((size_t)((2 + 2 * R + 1) * nl), sizeof(double));
    double *r = mem, *w = mem + nl;
    double** V = (double**)malloc((size_t)(R + 1) * sizeof(double*));
    double** Z = (double**)malloc((size_t)R * sizeof(double*));
    for (i64 j = 0; j <= R; ++j) V[j] = mem + (2 + j) * nl;
    for (i64 j = 0; j < R; ++j) Z[j] = mem + (2 + R + 1 + j) * nl;
    double* H = (double*)calloc((size_t)((R + 1) * R), sizeof(double));
    double* cs = (double*)calloc((size_t)R, sizeof(double));
    double* sn = (double*)calloc((size_t)R, sizeof(double));
    double* g = (double*)calloc((size_t)R + 1, sizeof(double));
    double* proj = (double*)calloc((size_t)R + 2, sizeof(double));
    double* coef = (double*)calloc((size_t)R + 1, sizeof(double));
#define HH(row, col) H[(col) * (R + 1) + (row)]
    true_residual(m, b, x, r, w, res);
    const double bnorm = norm_r(n, b, res), r0 = norm_r(n, r, res);
    const double thr = threshold_of(bnorm, o);
    res->initial_residual_norm = r0;
    set_residuals(res, r0, r0, bnorm);
    if (!isfinite(r0) || !isfinite(thr)) { breakdown(res, BR_NONFINITE); goto done; }
    if (r0 <= thr) { res->status = ST_CONVERGED; goto done; }
    while (res->iterations < o->maximum_iterations) {
        const double beta = norm_r(n, r, res);
        for (i64 i = 0; i < n; ++i) V[0][i] = r[i] / beta;
        memset(H, 0, (size_t)((R + 1) * R) * sizeof(double));
        memset(g, 0, (size_t)(R + 1) * sizeof(double));
        g[0] = beta;
        i64 cols = 0;
        int arnoldi_breakdown = 0;
        for (; cols < R && res->iterations < o->maximum_iterations; ++cols, ++res->iterations) {
            pc_apply(m, p, V[cols], Z[cols], res);
            op_apply(m, Z[cols], w, res);
            const i64 k = cols + 1;
            for (i64 row = 0; row < k; ++row) proj[row] = orc_dot(n, w, V[row]);
            proj[k] = orc_dot(n, w, w);
            res->global_reductions++;
            const double original = proj[k];
            double projected = original;
            for (i64 row = 0; row < k; ++row) {
                HH(row, cols) = proj[row];
                const double a = -HH(row, cols);
                for (i64 i = 0; i < n; ++i) w[i] += a * V[row][i];
                projected -= HH(row, cols) * HH(row, cols);
            }
            const double nonneg = projected > 0 ? projected : 0.0;
            const int forced = o->gmres_orthogonalization == 0;
            const int adaptive = o->gmres_orthogonalization == 1 && (projected <= 0 || nonneg < 0.5 * original);
            double nsq = nonneg;
            if (forced || adaptive) {
                for (i64 row = 0; row < k; ++row) proj[row] = orc_dot(n, w, V[row]);
                proj[k] = orc_dot(n, w, w);
                res->global_reductions++;
                res->reorthogonalizations++;
                nsq = proj[k];
                for (i64 row = 0; row < k; ++row) {
                    const double corr = proj[row];
                    HH(row, cols) += corr;
                    const double a = -corr;
                    for (i64 i = 0; i < n; ++i) w[i] += a * V[row][i];
                    nsq -= corr * corr;
                }
            }
            if (original < DBL_MIN || !isfinite(nsq) || nsq <= DBL_EPSILON * original
                || (nsq > 0 && nsq < DBL_MIN)) {
                HH(cols + 1, cols) = norm_r(n, w, res);
                res->arnoldi_norm_verifications++;
            } else {
                HH(cols + 1, cols) = sqrt(nsq > 0 ? nsq : 0.0);
            }
            if (!isfinite(HH(cols + 1, cols))) { breakdown(res, BR_NONFINITE); goto done; }
            double cscale = 0;
            for (i64 row = 0; row <= cols + 1; ++row) if (fabs(HH(row, cols)) > cscale) cscale = fabs(HH(row, cols));
            if (HH(cols + 1, cols) > o->breakdown_tolerance * cscale) {
                const double inv = 1.0 / HH(cols + 1, cols);
                for (i64 i = 0; i < n; ++i) V[cols + 1][i] = w[i];
                for (i64 i = 0; i < n; ++i) V[cols + 1][i] *= inv;
            } else {
                arnoldi_breakdown = 1;
            }
            for (i64 row = 0; row < cols; ++row) {
                const double first = cs[row] * HH(row, cols) + sn[row] * HH(row + 1, cols);
                HH(row + 1, cols) = -sn[row] * HH(row, cols) + cs[row] * HH(row + 1, cols);
                HH(row, cols) = first;
            }
            const double den = hypot(HH(cols, cols), HH(cols + 1, cols));
            if (!isfinite(den)) { breakdown(res, BR_NONFINITE); goto done; }
            if (den == 0) { arnoldi_breakdown = 1; cs[cols] = 1; sn[cols] = 0; }
            else { cs[cols] = HH(cols, cols) / den; sn[cols] = HH(cols + 1, cols) / den; }
            HH(cols, cols) = cs[cols] * HH(cols, cols) + sn[cols] * HH(cols + 1, cols);
            HH(cols + 1, cols) = 0;
            g[cols + 1] = -sn[cols] * g[cols];
            g[cols] *= cs[cols];
            const double est = fabs(g[cols + 1]);
            res->recursive_residual_norm = est;
            if (est <= thr || arnoldi_breakdown) { ++cols; ++res->iterations; break; }
        }
        memset(coef, 0, (size_t)(R + 1) * sizeof(double));
        for (i64 rv = cols - 1; rv >= 0; --rv) {
            double val = g[rv];
            for (i64 c = rv + 1; c < cols; ++c) val -= HH(rv, c) * coef[c];
            double cscale = 0;
            for (i64 row = 0; row <= rv; ++row) if (fabs(HH(row, rv)) > cscale) cscale = fabs(HH(row, rv));
            if (fabs(HH(rv, rv)) <= o->breakdown_tolerance * cscale) { breakdown(res, BR_SINGULAR); goto done; }
            coef[rv] = val / HH(rv, rv);
        }
        gmres_update(n, x, Z, coef, cols, x);
        true_residual(m, b, x, r, w, res);
        const double tn = norm_r(n, r, res);
        set_residuals(res, res->recursive_residual_norm, tn, bnorm);
        if (!isfinite(tn)) { breakdown(res, BR_NONFINITE); goto done; }
        if (tn <= thr) { res->status = ST_CONVERGED; goto done; }
        if (arnoldi_breakdown && !(tn < beta)) { breakdown(res, BR_ARNOLDI); goto done; }
    }
    res->status = ST_MAXIT;
done:
#undef HH
    free(mem); free(V); free(Z); free(H); free(cs); free(sn); free(g); free(proj); free(coef);
}

/* ------------------------------------------------------- dense-block ILU(0)
 * No counterpart in the reference (its ILU exists for component-diagonal
 * BlockCsrMatrix only, preconditioner.hpp:257).  Restated here as the checker
 * of the device's block factorisation, with the device's operation order:
 *   pattern   : ILU(0) of the block graph (sorted local columns, as
 *               preconditioner.hpp:373-427 with k = 0);
 *   factorise : per row, for each lower block l (pivot p, ascending column):
 *               L_l = A_l * Dinv_p, then A_t -= L_l * U_pu for every upper
 *               block u of row p whose column is present in the row;
 *               Dinv_r = inverse of the final diagonal block (Gauss-Jordan,
 *               partial pivoting, |pivot| <= 64 eps is a zero pivot);
 *   apply     : y_r = b_r - sum_l L_l y_col, x_r = Dinv_r (y_r - sum_u U_u x_col),
 *               each block product accumulated from +0 over j ascending. */
typedef struct {
    i64 owned, bs, entries;
    i64 *rp, *ci, *diagpos, *src;
    double *val, *dinv;   /* entries*bs*bs, owned*bs*bs */
} orc_block_ilu;

/* out = a (bs x bs) * b (bs x bs), row-major, sums from +0 in j order. */
static void block_mul(i64 bs, const double* a, const double* b, double* out)
{
    for (i64 i = 0; i < bs; ++i)
        for (i64 k = 0; k < bs; ++k) {
            double s = 0.0;
            for (i64 j = 0; j < bs; ++j) s += a[i * bs + j] * b[j * bs + k];
            out[i * bs + k] = s;
        }
}

/* Gauss-Jordan inverse with partial pivoting; returns 0 on a zero pivot. */
static int block_inverse(i64 bs, const double* a, double* inv)
{
    double m[64], r[64];
    for (i64 i = 0; i < bs * bs; ++i) { m[i] = a[i]; r[i] = 0.0; }
    for (i64 i = 0; i < bs; ++i) r[i * bs + i] = 1.0;
    for (i64 c = 0; c < bs; ++c) {
        i64 p = c;
        for (i64 i = c + 1; i < bs; ++i) if (fabs(m[i * bs + c]) > fabs(m[p * bs + c])) p = i;
        if (!isfinite(m[p * bs + c]) || fabs(m[p * bs + c]) <= 64.0 * DBL_EPSILON) return 0;
        if (p != c)
            for (i64 j = 0; j < bs; ++j) {
                double t = m[c * bs + j]; m[c * bs + j] = m[p * bs + j]; m[p * bs + j] = t;
                t = r[c * bs + j]; r[c * bs + j] = r[p * bs + j]; r[p * bs + j] = t;
            }
        const double piv = m[c * bs + c];
        for (i64 j = 0; j < bs; ++j) { m[c * bs + j] /= piv; r[c * bs + j] /= piv; }
        for (i64 i = 0; i < bs; ++i) {
            if (i == c) continue;
            const double f = m[i * bs + c];
            for (i64 j = 0; j < bs; ++j) { m[i * bs + j] -= f * m[c * bs + j]; r[i * bs + j] -= f * r[c * bs + j]; }
        }
    }
    for (i64 i = 0; i < bs * bs; ++i) inv[i] = r[i];
    return 1;
}

static i64 ilu_find_block(const orc_block_ilu* h, i64 r, i64 col)
{
    for (i64 e = h->rp[r]; e < h->rp[r + 1]; ++e)
        if (h->ci[e] == col) return e;
    return -1;
}

orc_block_ilu* orc_block_ilu_create(i64 owned, i64 bs, const i64* rp, const i64* ci, const double* v, int* status)
{
    int st = 0;
    orc_ilu* pat = orc_ilu_create(owned, 1, rp, ci, v /* unused values */, 0, &st);
    orc_block_ilu* h = (orc_block_ilu*)calloc(1, sizeof(orc_block_ilu));
    h->owned = owned; h->bs = bs;
    /* orc_ilu_create factorises bs=1 values too; only a pattern failure counts here. */
    if (st == ORC_INVALID) { *status = st; orc_ilu_destroy(pat); return h; }
    h->entries = pat->entries;
    h->rp = pat->rp; h->ci = pat->ci; h->diagpos = pat->diagpos; h->src = pat->src;
    pat->rp = pat->ci = pat->diagpos = pat->src = NULL;
    orc_ilu_destroy(pat);
    const i64 b2 = bs * bs;
    h->val = (double*)calloc((size_t)(h->entries * b2) + 1, sizeof(double));
    h->dinv = (double*)calloc((size_t)(owned * b2) + 1, sizeof(double));
    for (i64 e = 0; e < h->entries; ++e)
        if (h->src[e] >= 0) memcpy(h->val + e * b2, v + h->src[e] * b2, (size_t)b2 * sizeof(double));
    double tmp[64], lu[64];
    *status = ORC_OK;
    for (i64 r = 0; r < owned; ++r) {
        for (i64 l = h->rp[r]; l < h->diagpos[r]; ++l) {
            const i64 p = h->ci[l];
            block_mul(bs, h->val + l * b2, h->dinv + p * b2, tmp);
            memcpy(h->val + l * b2, tmp, (size_t)b2 * sizeof(double));
            for (i64 u = h->diagpos[p] + 1; u < h->rp[p + 1]; ++u) {
                const i64 t = ilu_find_block(h, r, h->ci[u]);
                if (t < 0) continue;
                block_mul(bs, h->val + l * b2, h->val + u * b2, lu);
                for (i64 k = 0; k < b2; ++k) h->val[t * b2 + k] -= lu[k];
            }
        }
        if (!block_inverse(bs, h->val + h->diagpos[r] * b2, h->dinv + r * b2)) { *status = ORC_ZERO_PIVOT; return h; }
    }
    return h;
}

void orc_block_ilu_apply(const orc_block_ilu* h, const double* in, double* out)
{
    const i64 bs = h->bs, b2 = bs * bs;
    double* y = (double*)malloc((size_t)(h->owned * bs) * sizeof(double));
    for (i64 r = 0; r < h->owned; ++r) {
        for (i64 i = 0; i < bs; ++i) {
            double acc = in[r * bs + i];
            for (i64 l = h->rp[r]; l < h->diagpos[r]; ++l) {
                const double* L = h->val + l * b2;
                const double* yc = y + h->ci[l] * bs;
                double s = 0.0;
                for (i64 j = 0; j < bs; ++j) s += L[i * bs + j] * yc[j];
                acc -= s;
            }
            y[r * bs + i] = acc;
        }
    }
    for (i64 r = h->owned - 1; r >= 0; --r) {
        double w[8];
        for (i64 i = 0; i < bs; ++i) {
            double acc = y[r * bs + i];
            for (i64 u = h->diagpos[r] + 1; u < h->rp[r + 1]; ++u) {
                const double* U = h->val + u * b2;
                const double* xc = out + h->ci[u] * bs;
                double s = 0.0;
                for (i64 j = 0; j < bs; ++j) s += U[i * bs + j] * xc[j];
                acc -= s;
            }
            w[i] = acc;
        }
        const double* D = h->dinv + r * b2;
        for (i64 i = 0; i < bs; ++i) {
            double s = 0.0;
            for (i64 j = 0; j < bs; ++j) s += D[i * bs + j] * w[j];
            out[r * bs + i] = s;
        }
    }
    free(y);
}

void orc_block_ilu_copy(const orc_block_ilu* h, double* val, double* dinv)
{
    const i64 b2 = h->bs * h->bs;
    if (val) memcpy(val, h->val, (size_t)(h->entries * b2) * sizeof(double));
    if (dinv) memcpy(dinv, h->dinv, (size_t)(h->owned * b2) * sizeof(double));
}

i64 orc_block_ilu_entries(const orc_block_ilu* h) { return h->entries; }

void orc_block_ilu_destroy(orc_block_ilu* h)
{
    if (!h) return;
    free(h->rp); free(h->ci); free(h->diagpos); free(h->src); free(h->val); free(h->dinv); free(h);
}
