/* ORACLE (test infrastructure only; never linked into the product).
 *
 * Fill-reducing column ordering, restated from ESPice
 * src/solver/order.zig: block triangular form by iterative Tarjan
 * (`blocks`, order.zig:154-235), AMD per non-singleton block (`amd`,
 * order.zig:375-692) or the natural order when its Cholesky count is
 * smaller (`order`, order.zig:78-147; `cholCount` order.zig:251-311).
 * Scratch comes from one caller-sized u32 slab (`Ws`, order.zig:18-57;
 * `wsSize` order.zig:67-69) so that OutOfWorkspace happens exactly where
 * the reference would raise it. The algorithm steps, the slab sizes and
 * the tie rules must stay the same as the reference's for the column order
 * to be bit-exact; the code is a plain C restatement.
 */
#include "oracle.h"

#include <stdlib.h>
#include <string.h>
#include <math.h>

#define NONE 0xFFFFFFFFu

typedef struct {
    uint32_t *buf;
    size_t len;
    size_t used;
} ws_t;

/* order.zig:31-37 */
static uint32_t *ws_alloc(ws_t *w, size_t m) {
    if (w->used + m > w->len) return NULL;
    uint32_t *s = w->buf + w->used;
    w->used += m;
    return s;
}

static uint32_t *ws_alloc_set(ws_t *w, size_t m, uint32_t fill) {
    uint32_t *s = ws_alloc(w, m);
    if (!s) return NULL;
    for (size_t i = 0; i < m; i++) s[i] = fill;
    return s;
}

size_t orc_ws_size(size_t n, size_t nnz) { return 48 * n + 8 * nnz + 64; }

#define ALLOC(dst, w, m)                          \
    do {                                          \
        (dst) = ws_alloc((w), (m));               \
        if (!(dst)) { (w)->used = base; return -1; } \
    } while (0)
#define ALLOC_SET(dst, w, m, f)                   \
    do {                                          \
        (dst) = ws_alloc_set((w), (m), (f));      \
        if (!(dst)) { (w)->used = base; return -1; } \
    } while (0)

/* Tarjan SCC, sink block first: order.zig:154-235. Returns the block count
 * or -1 on OutOfWorkspace. */
static int64_t blocks(uint32_t n, const uint32_t *col_ptr, const uint32_t *row_idx,
                      uint32_t *emit, uint32_t *block_ptr, ws_t *ws) {
    size_t base = ws->used;
    uint32_t *num, *low, *on, *scc_stack, *frame_v, *frame_p;
    ALLOC_SET(num, ws, n, NONE);
    ALLOC(low, ws, n);
    ALLOC_SET(on, ws, n, 0);
    ALLOC(scc_stack, ws, n);
    ALLOC(frame_v, ws, n);
    ALLOC(frame_p, ws, n);
    uint32_t sp = 0, fp = 0, counter = 0, no = 0, nb = 0;
    block_ptr[0] = 0;
    for (uint32_t root = 0; root < n; root++) {
        if (num[root] != NONE) continue;
        num[root] = counter;
        low[root] = counter;
        counter++;
        scc_stack[sp++] = root;
        on[root] = 1;
        frame_v[fp] = root;
        frame_p[fp] = col_ptr[root];
        fp++;
        while (fp > 0) {
            uint32_t v = frame_v[fp - 1];
            if (frame_p[fp - 1] < col_ptr[v + 1]) {
                uint32_t child = row_idx[frame_p[fp - 1]];
                frame_p[fp - 1]++;
                if (child == v) continue;
                if (num[child] == NONE) {
                    num[child] = counter;
                    low[child] = counter;
                    counter++;
                    scc_stack[sp++] = child;
                    on[child] = 1;
                    frame_v[fp] = child;
                    frame_p[fp] = col_ptr[child];
                    fp++;
                } else if (on[child]) {
                    if (num[child] < low[v]) low[v] = num[child];
                }
                continue;
            }
            if (low[v] == num[v]) {
                for (;;) {
                    sp--;
                    uint32_t m = scc_stack[sp];
                    on[m] = 0;
                    emit[no++] = m;
                    if (m == v) break;
                }
                nb++;
                block_ptr[nb] = no;
            }
            fp--;
            if (fp > 0) {
                uint32_t u = frame_v[fp - 1];
                if (low[v] < low[u]) low[u] = low[v];
            }
        }
    }
    ws->used = base;
    return nb;
}

/* Cholesky count of A + A^T under `perm`, capped: order.zig:251-311.
 * Returns UINT64_MAX on OutOfWorkspace. */
static uint64_t chol_count(uint32_t n, const uint32_t *col_ptr, const uint32_t *row_idx,
                           const uint32_t *perm, ws_t *ws, uint64_t cap) {
    size_t base = ws->used;
    uint32_t nnz = col_ptr[n];
    uint32_t *pinv = ws_alloc(ws, n);
    if (!pinv) { ws->used = base; return UINT64_MAX; }
    for (uint32_t k = 0; k < n; k++) pinv[perm[k]] = k;
    uint32_t *ptr = ws_alloc_set(ws, (size_t)n + 1, 0);
    uint32_t *lst = ptr ? ws_alloc(ws, nnz) : NULL;
    uint32_t *fill = lst ? ws_alloc(ws, n) : NULL;
    uint32_t *parent = fill ? ws_alloc(ws, n) : NULL;
    if (!parent) { ws->used = base; return UINT64_MAX; }
    for (uint32_t j = 0; j < n; j++)
        for (uint32_t p = col_ptr[j]; p < col_ptr[j + 1]; p++) {
            uint32_t a = pinv[row_idx[p]], b = pinv[j];
            if (a != b) ptr[(a > b ? a : b) + 1]++;
        }
    for (uint32_t k = 1; k <= n; k++) ptr[k] += ptr[k - 1];
    memcpy(fill, ptr, sizeof(uint32_t) * n);
    for (uint32_t j = 0; j < n; j++)
        for (uint32_t p = col_ptr[j]; p < col_ptr[j + 1]; p++) {
            uint32_t a = pinv[row_idx[p]], b = pinv[j];
            if (a == b) continue;
            uint32_t hi = a > b ? a : b;
            lst[fill[hi]] = a > b ? b : a;
            fill[hi]++;
        }
    uint32_t *anc = fill;
    for (uint32_t k = 0; k < n; k++) {
        parent[k] = NONE;
        anc[k] = NONE;
        for (uint32_t t = ptr[k]; t < ptr[k + 1]; t++) {
            uint32_t i = lst[t];
            while (i != NONE && i < k) {
                uint32_t next = anc[i];
                anc[i] = k;
                if (next == NONE) parent[i] = k;
                i = next;
            }
        }
    }
    uint32_t *flag = anc;
    uint64_t count = 0;
    for (uint32_t k = 0; k < n; k++) {
        flag[k] = k;
        count++;
        for (uint32_t t = ptr[k]; t < ptr[k + 1]; t++) {
            uint32_t i = lst[t];
            while (flag[i] != k) {
                flag[i] = k;
                count++;
                i = parent[i];
            }
        }
        if (count >= cap) { ws->used = base; return count; }
    }
    ws->used = base;
    return count;
}

#define SPAN_TAG (1u << 31)

/* order.zig:321-344 */
static size_t compact(uint32_t *adj, size_t top, uint32_t *pe, const uint32_t *len, uint32_t n,
                      const uint32_t *live_a, const uint32_t *live_b, uint32_t *first) {
    for (uint32_t o = 0; o < n; o++) {
        if (len[o] == 0 || (live_a[o] == 0 && live_b[o] == 0)) continue;
        first[o] = adj[pe[o]];
        adj[pe[o]] = SPAN_TAG | o;
    }
    size_t dst = 0, src = 0;
    while (src < top) {
        if ((adj[src] & SPAN_TAG) == 0) { src++; continue; }
        uint32_t o = adj[src] & ~SPAN_TAG;
        uint32_t l = len[o];
        adj[dst] = first[o];
        memmove(adj + dst + 1, adj + src + 1, sizeof(uint32_t) * (l - 1));
        pe[o] = (uint32_t)dst;
        dst += l;
        src += l;
    }
    return dst;
}

typedef struct { uint32_t *head, *next, *prev; } deglists;

static void dl_insert(deglists *s, uint32_t d, uint32_t i) {
    s->next[i] = s->head[d];
    s->prev[i] = NONE;
    if (s->head[d] != NONE) s->prev[s->head[d]] = i;
    s->head[d] = i;
}

static void dl_remove(deglists *s, uint32_t d, uint32_t i) {
    if (s->prev[i] != NONE) s->next[s->prev[i]] = s->next[i];
    else s->head[d] = s->next[i];
    if (s->next[i] != NONE) s->prev[s->next[i]] = s->prev[i];
}

/* order.zig:696-719 */
static int same_adj(const uint32_t *va, const uint32_t *va_pe, const uint32_t *va_len,
                    const uint32_t *ea, const uint32_t *ea_pe, const uint32_t *ea_len,
                    uint32_t *mark, uint32_t *era, uint32_t i, uint32_t j) {
    if (va_len[i] != va_len[j] || ea_len[i] != ea_len[j]) return 0;
    const uint32_t *adjs[2] = {va, ea};
    const uint32_t *pos[2] = {va_pe, ea_pe};
    const uint32_t *len[2] = {va_len, ea_len};
    for (int t = 0; t < 2; t++) {
        *era += 1;
        uint32_t m = *era;
        for (uint32_t k = 0; k < len[t][i]; k++) mark[adjs[t][pos[t][i] + k]] = m;
        for (uint32_t k = 0; k < len[t][j]; k++)
            if (mark[adjs[t][pos[t][j] + k]] != m) return 0;
    }
    return 1;
}

static uint32_t isqrt_u32(uint32_t n) {
    /* std.math.sqrt on an integer: floor(sqrt(n)). */
    uint32_t r = (uint32_t)sqrt((double)n);
    while ((uint64_t)r * r > n) r--;
    while ((uint64_t)(r + 1) * (r + 1) <= n) r++;
    return r;
}

/* AMD on the symmetrized pattern: order.zig:375-692. 0 or -1. */
static int amd(uint32_t n, const uint32_t *col_ptr, const uint32_t *row_idx, uint32_t *q, ws_t *ws) {
    if (n == 0) return 0;
    size_t base = ws->used;
    uint32_t nnz = col_ptr[n];
    size_t va_cap = 4 * (size_t)nnz + 4 * (size_t)n + 16;
    size_t ea_cap = 8 * (size_t)n + (size_t)nnz;
    uint32_t *va, *va_pe, *va_len, *ea, *ea_pe, *ea_len, *ea_lim, *nv, *elem_alive, *esize, *deg, *w_buf;
    uint32_t *mark_arr, *wmark_arr, *hkey, *hhead, *hnext, *hbuckets, *mlink, *lp_buf, *touched, *first;
    deglists dl;
    ALLOC(va, ws, va_cap);
    ALLOC(va_pe, ws, n);
    ALLOC(va_len, ws, n);
    ALLOC(ea, ws, ea_cap);
    ALLOC(ea_pe, ws, n);
    ALLOC_SET(ea_len, ws, n, 0);
    ALLOC(ea_lim, ws, n);
    ALLOC_SET(nv, ws, n, 1);
    ALLOC_SET(elem_alive, ws, n, 0);
    ALLOC(esize, ws, n);
    ALLOC(deg, ws, n);
    ALLOC(w_buf, ws, n);
    ALLOC_SET(mark_arr, ws, n, 0);
    ALLOC_SET(wmark_arr, ws, n, 0);
    uint32_t era = 0, erw = 0;
    ALLOC(hkey, ws, n);
    ALLOC_SET(hhead, ws, n, NONE);
    ALLOC(hnext, ws, n);
    ALLOC(hbuckets, ws, n);
    ALLOC_SET(mlink, ws, n, NONE);
    ALLOC(lp_buf, ws, n);
    ALLOC(touched, ws, n);
    ALLOC(first, ws, n);
    ALLOC_SET(dl.head, ws, (size_t)n + 1, NONE);
    ALLOC(dl.next, ws, n);
    ALLOC(dl.prev, ws, n);

    memset(deg, 0, sizeof(uint32_t) * n);
    for (uint32_t j = 0; j < n; j++)
        for (uint32_t p = col_ptr[j]; p < col_ptr[j + 1]; p++) {
            uint32_t r = row_idx[p];
            if (r == j) continue;
            deg[j]++;
            deg[r]++;
        }
    size_t va_free = 0;
    for (uint32_t i = 0; i < n; i++) {
        va_pe[i] = (uint32_t)va_free;
        va_free += deg[i];
    }
    memset(deg, 0, sizeof(uint32_t) * n);
    for (uint32_t j = 0; j < n; j++)
        for (uint32_t p = col_ptr[j]; p < col_ptr[j + 1]; p++) {
            uint32_t r = row_idx[p];
            if (r == j) continue;
            va[va_pe[j] + deg[j]] = r;
            deg[j]++;
            va[va_pe[r] + deg[r]] = j;
            deg[r]++;
        }
    memcpy(va_len, deg, sizeof(uint32_t) * n);
    for (uint32_t i = 0; i < n; i++) {
        era++;
        uint32_t wp = 0, s = va_pe[i];
        for (uint32_t k = 0; k < va_len[i]; k++) {
            uint32_t v = va[s + k];
            if (mark_arr[v] != era) {
                mark_arr[v] = era;
                va[s + wp++] = v;
            }
        }
        va_len[i] = wp;
    }

    uint32_t isq = isqrt_u32(n);
    uint32_t dense_thresh = 10 * isq > 16 ? 10 * isq : 16;
    uint32_t ndense = 0;
    for (uint32_t i = 0; i < n; i++) ndense += va_len[i] >= dense_thresh;
    uint32_t dense_start = n - ndense;
    {
        uint32_t di = 0;
        for (uint32_t i = 0; i < n; i++)
            if (va_len[i] >= dense_thresh) {
                nv[i] = 0;
                lp_buf[dense_start + di++] = i;
            }
    }
    if (ndense > 0) {
        for (uint32_t i = 0; i < n; i++) {
            if (nv[i] == 0) continue;
            uint32_t wp = 0, s = va_pe[i];
            for (uint32_t k = 0; k < va_len[i]; k++) {
                uint32_t v = va[s + k];
                if (nv[v] != 0) va[s + wp++] = v;
            }
            va_len[i] = wp;
        }
    }
    size_t ea_free = 0;
    for (uint32_t i = 0; i < n; i++) {
        ea_pe[i] = (uint32_t)ea_free;
        ea_lim[i] = 4;
        ea_free += 4;
    }
    for (uint32_t i = 0; i < n; i++) {
        if (nv[i] == 0) continue;
        deg[i] = va_len[i];
        dl_insert(&dl, deg[i], i);
    }
    uint32_t n_amd = n - ndense, mindeg = 0, k = 0;
    while (k < n_amd) {
        while (dl.head[mindeg] == NONE) mindeg++;
        uint32_t p = dl.head[mindeg];
        dl_remove(&dl, deg[p], p);
        era++;
        mark_arr[p] = era;
        uint32_t nlp = 0;
        for (uint32_t t = 0; t < va_len[p]; t++) {
            uint32_t v = va[va_pe[p] + t];
            if (nv[v] != 0 && mark_arr[v] != era) {
                mark_arr[v] = era;
                lp_buf[nlp++] = v;
            }
        }
        for (uint32_t t = 0; t < ea_len[p]; t++) {
            uint32_t e = ea[ea_pe[p] + t];
            if (elem_alive[e] == 0) continue;
            for (uint32_t s2 = 0; s2 < va_len[e]; s2++) {
                uint32_t v = va[va_pe[e] + s2];
                if (nv[v] != 0 && mark_arr[v] != era) {
                    mark_arr[v] = era;
                    lp_buf[nlp++] = v;
                }
            }
            elem_alive[e] = 0;
        }
        uint32_t nvpiv = nv[p];
        nv[p] = 0;
        elem_alive[p] = 1;
        if (va_free + nlp > va_cap) {
            va_len[p] = 0;
            va_free = compact(va, va_free, va_pe, va_len, n, nv, elem_alive, first);
            if (va_free + nlp > va_cap) { ws->used = base; return -1; }
        }
        va_pe[p] = (uint32_t)va_free;
        va_len[p] = nlp;
        memcpy(va + va_free, lp_buf, sizeof(uint32_t) * nlp);
        va_free += nlp;

        uint32_t lpsize = 0;
        for (uint32_t t = 0; t < nlp; t++) lpsize += nv[lp_buf[t]];
        esize[p] = lpsize;
        for (uint32_t t = 0; t < nlp; t++) dl_remove(&dl, deg[lp_buf[t]], lp_buf[t]);

        erw++;
        uint32_t ntouched = 0;
        for (uint32_t t = 0; t < nlp; t++) {
            uint32_t i = lp_buf[t];
            for (uint32_t s2 = 0; s2 < ea_len[i]; s2++) {
                uint32_t e = ea[ea_pe[i] + s2];
                if (elem_alive[e] == 0) continue;
                if (wmark_arr[e] != erw) {
                    wmark_arr[e] = erw;
                    w_buf[e] = esize[e];
                    touched[ntouched++] = e;
                }
                w_buf[e] -= (w_buf[e] < nv[i] ? w_buf[e] : nv[i]);
            }
        }
        for (uint32_t t = 0; t < ntouched; t++)
            if (w_buf[touched[t]] == 0) elem_alive[touched[t]] = 0;
        for (uint32_t t = 0; t < nlp; t++) {
            uint32_t i = lp_buf[t];
            uint32_t esum = 0, ewp = 0;
            for (uint32_t s2 = 0; s2 < ea_len[i]; s2++) {
                uint32_t e = ea[ea_pe[i] + s2];
                if (elem_alive[e] != 0 && e != p) {
                    ea[ea_pe[i] + ewp++] = e;
                    esum += w_buf[e];
                }
            }
            if (ewp < ea_lim[i]) {
                ea[ea_pe[i] + ewp] = p;
            } else {
                uint32_t nc = (ewp + 1) * 2;
                if (ea_free + nc > ea_cap) {
                    ea_len[i] = ewp;
                    ea_free = compact(ea, ea_free, ea_pe, ea_len, n, nv, nv, first);
                    for (uint32_t o = 0; o < n; o++) ea_lim[o] = ea_len[o];
                    if (ea_free + nc > ea_cap) { ws->used = base; return -1; }
                }
                memmove(ea + ea_free, ea + ea_pe[i], sizeof(uint32_t) * ewp);
                ea[ea_free + ewp] = p;
                ea_pe[i] = (uint32_t)ea_free;
                ea_lim[i] = nc;
                ea_free += nc;
            }
            ea_len[i] = ewp + 1;
            uint32_t asum = 0, vwp = 0;
            for (uint32_t s2 = 0; s2 < va_len[i]; s2++) {
                uint32_t v = va[va_pe[i] + s2];
                if (nv[v] != 0 && mark_arr[v] != era) {
                    va[va_pe[i] + vwp++] = v;
                    asum += nv[v];
                }
            }
            va_len[i] = vwp;
            uint32_t cap = n_amd - k - nvpiv;
            uint32_t d = asum + (lpsize - nv[i]) + esum;
            deg[i] = d < cap ? d : cap;
        }
        uint32_t nhb = 0;
        for (uint32_t t = 0; t < nlp; t++) {
            uint32_t i = lp_buf[t];
            if (nv[i] == 0) continue;
            uint32_t h = 0;
            for (uint32_t s2 = 0; s2 < va_len[i]; s2++) h += va[va_pe[i] + s2];
            for (uint32_t s2 = 0; s2 < ea_len[i]; s2++) h += ea[ea_pe[i] + s2];
            hkey[i] = h;
            uint32_t b = h % n;
            if (hhead[b] == NONE) hbuckets[nhb++] = b;
            hnext[i] = hhead[b];
            hhead[b] = i;
        }
        for (uint32_t hb = 0; hb < nhb; hb++) {
            uint32_t b = hbuckets[hb];
            for (uint32_t i = hhead[b]; i != NONE; i = hnext[i]) {
                if (nv[i] == 0) continue;
                for (uint32_t j = hnext[i]; j != NONE; j = hnext[j]) {
                    if (nv[j] == 0 || hkey[j] != hkey[i]) continue;
                    if (!same_adj(va, va_pe, va_len, ea, ea_pe, ea_len, mark_arr, &era, i, j)) continue;
                    deg[i] -= (deg[i] < nv[j] ? deg[i] : nv[j]);
                    nv[i] += nv[j];
                    nv[j] = 0;
                    uint32_t tail = j;
                    while (mlink[tail] != NONE) tail = mlink[tail];
                    mlink[tail] = mlink[i];
                    mlink[i] = j;
                }
            }
            hhead[b] = NONE;
        }
        for (uint32_t t = 0; t < nlp; t++) {
            uint32_t i = lp_buf[t];
            if (nv[i] == 0) continue;
            dl_insert(&dl, deg[i], i);
            if (deg[i] < mindeg) mindeg = deg[i];
        }
        q[k++] = p;
        for (uint32_t mb = mlink[p]; mb != NONE; mb = mlink[mb]) q[k++] = mb;
    }
    memcpy(q + k, lp_buf + dense_start, sizeof(uint32_t) * ndense);
    ws->used = base;
    return 0;
}

static int cmp_u32(const void *a, const void *b) {
    uint32_t x = *(const uint32_t *)a, y = *(const uint32_t *)b;
    return x < y ? -1 : x > y;
}

/* order.zig:78-147. */
static int order_ws(uint32_t n, const uint32_t *col_ptr, const uint32_t *row_idx, uint32_t *q, ws_t *ws) {
    if (n == 0) return 0;
    size_t base = ws->used;
    uint32_t *emit, *block_ptr, *blk_of, *loc;
    ALLOC(emit, ws, n);
    ALLOC(block_ptr, ws, (size_t)n + 1);
    int64_t nb = blocks(n, col_ptr, row_idx, emit, block_ptr, ws);
    if (nb < 0) { ws->used = base; return -1; }
    ALLOC(blk_of, ws, n);
    ALLOC(loc, ws, n);
    for (uint32_t b = 0; b < nb; b++)
        for (uint32_t i = block_ptr[b], li = 0; i < block_ptr[b + 1]; i++, li++) {
            blk_of[emit[i]] = b;
            loc[emit[i]] = li;
        }
    for (uint32_t b = 0; b < nb; b++) {
        uint32_t lo = block_ptr[b], hi = block_ptr[b + 1], bs = hi - lo;
        const uint32_t *verts = emit + lo;
        if (bs == 1) { q[lo] = verts[0]; continue; }
        size_t blk_mark = ws->used;
        uint32_t *sub_cp, *sub_ri, *sub_q, *nat;
        ALLOC(sub_cp, ws, (size_t)bs + 1);
        uint32_t sub_nnz = 0;
        sub_cp[0] = 0;
        for (uint32_t j = 0; j < bs; j++) {
            uint32_t v = verts[j];
            for (uint32_t p = col_ptr[v]; p < col_ptr[v + 1]; p++) sub_nnz += blk_of[row_idx[p]] == b;
            sub_cp[j + 1] = sub_nnz;
        }
        ALLOC(sub_ri, ws, sub_nnz);
        uint32_t w = 0;
        for (uint32_t j = 0; j < bs; j++) {
            uint32_t v = verts[j];
            for (uint32_t p = col_ptr[v]; p < col_ptr[v + 1]; p++) {
                uint32_t r = row_idx[p];
                if (blk_of[r] == b) sub_ri[w++] = loc[r];
            }
        }
        ALLOC(sub_q, ws, bs);
        if (amd(bs, sub_cp, sub_ri, sub_q, ws) != 0) { ws->used = base; return -1; }
        ALLOC(nat, ws, bs);
        memcpy(nat, verts, sizeof(uint32_t) * bs);
        qsort(nat, bs, sizeof(uint32_t), cmp_u32);
        for (uint32_t i = 0; i < bs; i++) nat[i] = loc[nat[i]];
        uint64_t amd_count = chol_count(bs, sub_cp, sub_ri, sub_q, ws, UINT64_MAX);
        if (amd_count == UINT64_MAX) { ws->used = base; return -1; }
        uint64_t nat_count = chol_count(bs, sub_cp, sub_ri, nat, ws, amd_count);
        if (nat_count == UINT64_MAX) { ws->used = base; return -1; }
        const uint32_t *ord = nat_count < amd_count ? nat : sub_q;
        for (uint32_t i = 0; i < bs; i++) q[lo + i] = verts[ord[i]];
        ws->used = blk_mark;
    }
    ws->used = base;
    return 0;
}

int orc_order_ws(uint32_t n, const uint32_t *col_ptr, const uint32_t *row_idx, uint32_t *q,
                 uint32_t *slab, size_t slab_len) {
    ws_t ws = {slab, slab_len, 0};
    return order_ws(n, col_ptr, row_idx, q, &ws);
}

int orc_amd_ws(uint32_t n, const uint32_t *col_ptr, const uint32_t *row_idx, uint32_t *q,
               uint32_t *slab, size_t slab_len) {
    ws_t ws = {slab, slab_len, 0};
    return amd(n, col_ptr, row_idx, q, &ws);
}

int orc_order(uint32_t n, const uint32_t *col_ptr, const uint32_t *row_idx, uint32_t *q) {
    size_t len = orc_ws_size(n, col_ptr[n]);
    uint32_t *slab = (uint32_t *)malloc(sizeof(uint32_t) * (len ? len : 1));
    if (!slab) return -2;
    int r = orc_order_ws(n, col_ptr, row_idx, q, slab, len);
    free(slab);
    return r;
}

uint64_t orc_chol_count(uint32_t n, const uint32_t *col_ptr, const uint32_t *row_idx,
                        const uint32_t *perm, uint64_t cap) {
    size_t len = orc_ws_size(n, col_ptr[n]);
    uint32_t *slab = (uint32_t *)malloc(sizeof(uint32_t) * (len ? len : 1));
    ws_t ws = {slab, len, 0};
    uint64_t r = chol_count(n, col_ptr, row_idx, perm, &ws, cap);
    free(slab);
    return r;
}

/* order.zig:241-244 */
uint64_t orc_diag_fill(uint32_t n, const uint32_t *col_ptr, const uint32_t *row_idx, const uint32_t *q) {
    return 2 * (orc_chol_count(n, col_ptr, row_idx, q, UINT64_MAX) - n);
}
