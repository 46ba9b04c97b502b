// Host symbolic analysis for the lane tapes. See tape.h.
//
// The column order is the reference's algorithm step for step, because the
// tape must be bit-exact with it: Tarjan's SCC blocks sink first
// (order.zig:154-235), AMD per non-singleton block with approximate external
// degrees, aggressive absorption, hashed supervariables and dense-row
// deferral (order.zig:375-692), and the natural order where its Cholesky
// count (order.zig:251-311) is smaller (order.zig:78-147). The same holds for
// the pivot sequence of the lead lane's factor (sparse_lu.zig:337-663,
// supernodal walk :754-910).
#include "tape.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>

namespace espl {
namespace {

// A bump slab with the reference's capacity, so OutOfWorkspace strikes at
// the same pattern sizes.
struct Slab {
    std::vector<uint32_t> buf;
    size_t used = 0;
    explicit Slab(size_t len) : buf(len + 1), cap(len) {}
    size_t cap;
    uint32_t* take(size_t m) {
        if (used + m > cap) return nullptr;
        uint32_t* s = buf.data() + used;
        used += m;
        return s;
    }
    uint32_t* take(size_t m, uint32_t fill) {
        uint32_t* s = take(m);
        if (s) std::fill(s, s + m, fill);
        return s;
    }
};

size_t slab_words(size_t n, size_t nnz) { return 48 * n + 8 * nnz + 64; }

int64_t scc_blocks(uint32_t n, const uint32_t* cp, const uint32_t* ri, uint32_t* emit, uint32_t* bptr, Slab& ws) {
    size_t mark = ws.used;
    uint32_t* num = ws.take(n, kNone);
    uint32_t* low = ws.take(n);
    uint32_t* on = ws.take(n, 0);
    uint32_t* stk = ws.take(n);
    uint32_t* fv = ws.take(n);
    uint32_t* fpos = ws.take(n);
    if (!fpos) { ws.used = mark; return -1; }
    uint32_t sp = 0, fp = 0, counter = 0, no = 0, nb = 0;
    bptr[0] = 0;
    for (uint32_t root = 0; root < n; root++) {
        if (num[root] != kNone) continue;
        num[root] = low[root] = counter++;
        stk[sp++] = root;
        on[root] = 1;
        fv[fp] = root;
        fpos[fp] = cp[root];
        fp++;
        while (fp > 0) {
            uint32_t v = fv[fp - 1];
            if (fpos[fp - 1] < cp[v + 1]) {
                uint32_t ch = ri[fpos[fp - 1]++];
                if (ch == v) continue;
                if (num[ch] == kNone) {
                    num[ch] = low[ch] = counter++;
                    stk[sp++] = ch;
                    on[ch] = 1;
                    fv[fp] = ch;
                    fpos[fp] = cp[ch];
                    fp++;
                } else if (on[ch]) {
                    low[v] = std::min(low[v], num[ch]);
                }
                continue;
            }
            if (low[v] == num[v]) {
                for (;;) {
                    uint32_t m = stk[--sp];
                    on[m] = 0;
                    emit[no++] = m;
                    if (m == v) break;
                }
                bptr[++nb] = no;
            }
            fp--;
            if (fp > 0) low[fv[fp - 1]] = std::min(low[fv[fp - 1]], low[v]);
        }
    }
    ws.used = mark;
    return nb;
}

constexpr uint64_t kCountFail = std::numeric_limits<uint64_t>::max();

uint64_t chol_count(uint32_t n, const uint32_t* cp, const uint32_t* ri, const uint32_t* perm, Slab& ws, uint64_t cap) {
    size_t mark = ws.used;
    uint32_t nnz = cp[n];
    uint32_t* pinv = ws.take(n);
    uint32_t* ptr = pinv ? ws.take(size_t(n) + 1, 0) : nullptr;
    uint32_t* lst = ptr ? ws.take(nnz) : nullptr;
    uint32_t* fill = lst ? ws.take(n) : nullptr;
    uint32_t* parent = fill ? ws.take(n) : nullptr;
    if (!parent && n) { ws.used = mark; return kCountFail; }
    for (uint32_t k = 0; k < n; k++) pinv[perm[k]] = k;
    for (uint32_t j = 0; j < n; j++)
        for (uint32_t p = cp[j]; p < cp[j + 1]; p++) {
            uint32_t a = pinv[ri[p]], b = pinv[j];
            if (a != b) ptr[std::max(a, b) + 1]++;
        }
    for (uint32_t k = 1; k <= n; k++) ptr[k] += ptr[k - 1];
    std::memcpy(fill, ptr, sizeof(uint32_t) * n);
    for (uint32_t j = 0; j < n; j++)
        for (uint32_t p = cp[j]; p < cp[j + 1]; p++) {
            uint32_t a = pinv[ri[p]], b = pinv[j];
            if (a == b) continue;
            uint32_t hi = std::max(a, b);
            lst[fill[hi]++] = std::min(a, b);
        }
    uint32_t* anc = fill;
    for (uint32_t k = 0; k < n; k++) {
        parent[k] = anc[k] = kNone;
        for (uint32_t t = ptr[k]; t < ptr[k + 1]; t++)
            for (uint32_t i = lst[t]; i != kNone && i < k;) {
                uint32_t nx = anc[i];
                anc[i] = k;
                if (nx == kNone) parent[i] = k;
                i = nx;
            }
    }
    uint32_t* flag = anc;
    uint64_t count = 0;
    for (uint32_t k = 0; k < n; k++) {
        flag[k] = k;
        count++;
        for (uint32_t t = ptr[k]; t < ptr[k + 1]; t++)
            for (uint32_t i = lst[t]; flag[i] != k; i = parent[i]) {
                flag[i] = k;
                count++;
            }
        if (count >= cap) { ws.used = mark; return count; }
    }
    ws.used = mark;
    return count;
}

constexpr uint32_t kSpanTag = 1u << 31;

size_t compact_spans(uint32_t* adj, size_t top, uint32_t* pe, const uint32_t* len, uint32_t n, const uint32_t* la,
                     const uint32_t* lb, uint32_t* first) {
    for (uint32_t o = 0; o < n; o++) {
        if (len[o] == 0 || (la[o] == 0 && lb[o] == 0)) continue;
        first[o] = adj[pe[o]];
        adj[pe[o]] = kSpanTag | o;
    }
    size_t dst = 0, src = 0;
    while (src < top) {
        if (!(adj[src] & kSpanTag)) { src++; continue; }
        uint32_t o = adj[src] & ~kSpanTag;
        uint32_t l = len[o];
        adj[dst] = first[o];
        std::memmove(adj + dst + 1, adj + src + 1, sizeof(uint32_t) * (l - 1));
        pe[o] = uint32_t(dst);
        dst += l;
        src += l;
    }
    return dst;
}

bool same_adjacency(const uint32_t* va, const uint32_t* vpe, const uint32_t* vlen, const uint32_t* ea,
                    const uint32_t* epe, const uint32_t* elen, uint32_t* mark, uint32_t& era, uint32_t i, uint32_t j) {
    if (vlen[i] != vlen[j] || elen[i] != elen[j]) return false;
    const uint32_t* adj[2] = {va, ea};
    const uint32_t* pos[2] = {vpe, epe};
    const uint32_t* len[2] = {vlen, elen};
    for (int t = 0; t < 2; t++) {
        uint32_t m = ++era;
        for (uint32_t k = 0; k < len[t][i]; k++) mark[adj[t][pos[t][i] + k]] = m;
        for (uint32_t k = 0; k < len[t][j]; k++)
            if (mark[adj[t][pos[t][j] + k]] != m) return false;
    }
    return true;
}

bool amd_order(uint32_t n, const uint32_t* cp, const uint32_t* ri, uint32_t* q, Slab& ws) {
    if (n == 0) return true;
    size_t mark0 = ws.used;
    uint32_t nnz = cp[n];
    size_t va_cap = 4 * size_t(nnz) + 4 * size_t(n) + 16, ea_cap = 8 * size_t(n) + nnz;
    uint32_t* va = ws.take(va_cap);
    uint32_t* vpe = ws.take(n);
    uint32_t* vlen = ws.take(n);
    uint32_t* ea = ws.take(ea_cap);
    uint32_t* epe = ws.take(n);
    uint32_t* elen = ws.take(n, 0);
    uint32_t* elim = ws.take(n);
    uint32_t* nv = ws.take(n, 1);
    uint32_t* alive = ws.take(n, 0);
    uint32_t* esize = ws.take(n);
    uint32_t* deg = ws.take(n);
    uint32_t* wb = ws.take(n);
    uint32_t* mk = ws.take(n, 0);
    uint32_t* wmk = ws.take(n, 0);
    uint32_t* hkey = ws.take(n);
    uint32_t* hhead = ws.take(n, kNone);
    uint32_t* hnext = ws.take(n);
    uint32_t* hbk = ws.take(n);
    uint32_t* mlink = ws.take(n, kNone);
    uint32_t* lpb = ws.take(n);
    uint32_t* touched = ws.take(n);
    uint32_t* first = ws.take(n);
    uint32_t* dhead = ws.take(size_t(n) + 1, kNone);
    uint32_t* dnext = ws.take(n);
    uint32_t* dprev = ws.take(n);
    if (!dprev) { ws.used = mark0; return false; }
    uint32_t era = 0, erw = 0;
    auto dins = [&](uint32_t d, uint32_t i) {
        dnext[i] = dhead[d];
        dprev[i] = kNone;
        if (dhead[d] != kNone) dprev[dhead[d]] = i;
        dhead[d] = i;
    };
    auto drem = [&](uint32_t d, uint32_t i) {
        if (dprev[i] != kNone) dnext[dprev[i]] = dnext[i];
        else dhead[d] = dnext[i];
        if (dnext[i] != kNone) dprev[dnext[i]] = dprev[i];
    };
    std::fill(deg, deg + n, 0);
    for (uint32_t j = 0; j < n; j++)
        for (uint32_t p = cp[j]; p < cp[j + 1]; p++)
            if (ri[p] != j) { deg[j]++; deg[ri[p]]++; }
    size_t vfree = 0;
    for (uint32_t i = 0; i < n; i++) { vpe[i] = uint32_t(vfree); vfree += deg[i]; }
    std::fill(deg, deg + n, 0);
    for (uint32_t j = 0; j < n; j++)
        for (uint32_t p = cp[j]; p < cp[j + 1]; p++) {
            uint32_t r = ri[p];
            if (r == j) continue;
            va[vpe[j] + deg[j]++] = r;
            va[vpe[r] + deg[r]++] = j;
        }
    std::memcpy(vlen, deg, sizeof(uint32_t) * n);
    for (uint32_t i = 0; i < n; i++) {
        era++;
        uint32_t wp = 0, s = vpe[i];
        for (uint32_t k = 0; k < vlen[i]; k++) {
            uint32_t v = va[s + k];
            if (mk[v] != era) { mk[v] = era; va[s + wp++] = v; }
        }
        vlen[i] = wp;
    }
    uint32_t isq = uint32_t(std::sqrt(double(n)));
    while (uint64_t(isq) * isq > n) isq--;
    while (uint64_t(isq + 1) * (isq + 1) <= n) isq++;
    uint32_t dthr = std::max<uint32_t>(16, 10 * isq);
    uint32_t ndense = 0;
    for (uint32_t i = 0; i < n; i++) ndense += vlen[i] >= dthr;
    uint32_t dstart = n - ndense;
    for (uint32_t i = 0, di = 0; i < n; i++)
        if (vlen[i] >= dthr) { nv[i] = 0; lpb[dstart + di++] = i; }
    if (ndense)
        for (uint32_t i = 0; i < n; i++) {
            if (!nv[i]) continue;
            uint32_t wp = 0, s = vpe[i];
            for (uint32_t k = 0; k < vlen[i]; k++)
                if (nv[va[s + k]]) va[s + wp++] = va[s + k];
            vlen[i] = wp;
        }
    size_t efree = 0;
    for (uint32_t i = 0; i < n; i++) { epe[i] = uint32_t(efree); elim[i] = 4; efree += 4; }
    for (uint32_t i = 0; i < n; i++)
        if (nv[i]) { deg[i] = vlen[i]; dins(deg[i], i); }
    uint32_t namd = n - ndense, mindeg = 0, k = 0;
    while (k < namd) {
        while (dhead[mindeg] == kNone) mindeg++;
        uint32_t p = dhead[mindeg];
        drem(deg[p], p);
        era++;
        mk[p] = era;
        uint32_t nlp = 0;
        for (uint32_t t = 0; t < vlen[p]; t++) {
            uint32_t v = va[vpe[p] + t];
            if (nv[v] && mk[v] != era) { mk[v] = era; lpb[nlp++] = v; }
        }
        for (uint32_t t = 0; t < elen[p]; t++) {
            uint32_t e = ea[epe[p] + t];
            if (!alive[e]) continue;
            for (uint32_t s2 = 0; s2 < vlen[e]; s2++) {
                uint32_t v = va[vpe[e] + s2];
                if (nv[v] && mk[v] != era) { mk[v] = era; lpb[nlp++] = v; }
            }
            alive[e] = 0;
        }
        uint32_t nvpiv = nv[p];
        nv[p] = 0;
        alive[p] = 1;
        if (vfree + nlp > va_cap) {
            vlen[p] = 0;
            vfree = compact_spans(va, vfree, vpe, vlen, n, nv, alive, first);
            if (vfree + nlp > va_cap) { ws.used = mark0; return false; }
        }
        vpe[p] = uint32_t(vfree);
        vlen[p] = nlp;
        std::memcpy(va + vfree, lpb, sizeof(uint32_t) * nlp);
        vfree += nlp;
        uint32_t lpsize = 0;
        for (uint32_t t = 0; t < nlp; t++) lpsize += nv[lpb[t]];
        esize[p] = lpsize;
        for (uint32_t t = 0; t < nlp; t++) drem(deg[lpb[t]], lpb[t]);
        erw++;
        uint32_t nt = 0;
        for (uint32_t t = 0; t < nlp; t++) {
            uint32_t i = lpb[t];
            for (uint32_t s2 = 0; s2 < elen[i]; s2++) {
                uint32_t e = ea[epe[i] + s2];
                if (!alive[e]) continue;
                if (wmk[e] != erw) { wmk[e] = erw; wb[e] = esize[e]; touched[nt++] = e; }
                wb[e] -= std::min(wb[e], nv[i]);
            }
        }
        for (uint32_t t = 0; t < nt; t++)
            if (wb[touched[t]] == 0) alive[touched[t]] = 0;
        for (uint32_t t = 0; t < nlp; t++) {
            uint32_t i = lpb[t];
            uint32_t esum = 0, ewp = 0;
            for (uint32_t s2 = 0; s2 < elen[i]; s2++) {
                uint32_t e = ea[epe[i] + s2];
                if (alive[e] && e != p) { ea[epe[i] + ewp++] = e; esum += wb[e]; }
            }
            if (ewp < elim[i]) {
                ea[epe[i] + ewp] = p;
            } else {
                uint32_t nc = (ewp + 1) * 2;
                if (efree + nc > ea_cap) {
                    elen[i] = ewp;
                    efree = compact_spans(ea, efree, epe, elen, n, nv, nv, first);
                    for (uint32_t o = 0; o < n; o++) elim[o] = elen[o];
                    if (efree + nc > ea_cap) { ws.used = mark0; return false; }
                }
                std::memmove(ea + efree, ea + epe[i], sizeof(uint32_t) * ewp);
                ea[efree + ewp] = p;
                epe[i] = uint32_t(efree);
                elim[i] = nc;
                efree += nc;
            }
            elen[i] = ewp + 1;
            uint32_t asum = 0, vwp = 0;
            for (uint32_t s2 = 0; s2 < vlen[i]; s2++) {
                uint32_t v = va[vpe[i] + s2];
                if (nv[v] && mk[v] != era) { va[vpe[i] + vwp++] = v; asum += nv[v]; }
            }
            vlen[i] = vwp;
            deg[i] = std::min(asum + (lpsize - nv[i]) + esum, namd - k - nvpiv);
        }
        uint32_t nhb = 0;
        for (uint32_t t = 0; t < nlp; t++) {
            uint32_t i = lpb[t];
            if (!nv[i]) continue;
            uint32_t h = 0;
            for (uint32_t s2 = 0; s2 < vlen[i]; s2++) h += va[vpe[i] + s2];
            for (uint32_t s2 = 0; s2 < elen[i]; s2++) h += ea[epe[i] + s2];
            hkey[i] = h;
            uint32_t b = h % n;
            if (hhead[b] == kNone) hbk[nhb++] = b;
            hnext[i] = hhead[b];
            hhead[b] = i;
        }
        for (uint32_t hb = 0; hb < nhb; hb++) {
            uint32_t b = hbk[hb];
            for (uint32_t i = hhead[b]; i != kNone; i = hnext[i]) {
                if (!nv[i]) continue;
                for (uint32_t j = hnext[i]; j != kNone; j = hnext[j]) {
                    if (!nv[j] || hkey[j] != hkey[i]) continue;
                    if (!same_adjacency(va, vpe, vlen, ea, epe, elen, mk, era, i, j)) continue;
                    deg[i] -= std::min(deg[i], nv[j]);
                    nv[i] += nv[j];
                    nv[j] = 0;
                    uint32_t tail = j;
                    while (mlink[tail] != kNone) tail = mlink[tail];
                    mlink[tail] = mlink[i];
                    mlink[i] = j;
                }
            }
            hhead[b] = kNone;
        }
        for (uint32_t t = 0; t < nlp; t++) {
            uint32_t i = lpb[t];
            if (!nv[i]) continue;
            dins(deg[i], i);
            mindeg = std::min(mindeg, deg[i]);
        }
        q[k++] = p;
        for (uint32_t mb = mlink[p]; mb != kNone; mb = mlink[mb]) q[k++] = mb;
    }
    std::memcpy(q + k, lpb + dstart, sizeof(uint32_t) * ndense);
    ws.used = mark0;
    return true;
}

bool order_in(uint32_t n, const uint32_t* cp, const uint32_t* ri, uint32_t* q, Slab& ws) {
    if (n == 0) return true;
    size_t mark0 = ws.used;
    uint32_t* emit = ws.take(n);
    uint32_t* bptr = emit ? ws.take(size_t(n) + 1) : nullptr;
    if (!bptr) { ws.used = mark0; return false; }
    int64_t nb = scc_blocks(n, cp, ri, emit, bptr, ws);
    if (nb < 0) { ws.used = mark0; return false; }
    uint32_t* blk = ws.take(n);
    uint32_t* loc = blk ? ws.take(n) : nullptr;
    if (!loc) { ws.used = mark0; return false; }
    for (uint32_t b = 0; b < uint32_t(nb); b++)
        for (uint32_t i = bptr[b], li = 0; i < bptr[b + 1]; i++, li++) { blk[emit[i]] = b; loc[emit[i]] = li; }
    for (uint32_t b = 0; b < uint32_t(nb); b++) {
        uint32_t lo = bptr[b], hi = bptr[b + 1], bs = hi - lo;
        const uint32_t* verts = emit + lo;
        if (bs == 1) { q[lo] = verts[0]; continue; }
        size_t bmark = ws.used;
        uint32_t* scp = ws.take(size_t(bs) + 1);
        if (!scp) { ws.used = mark0; return false; }
        uint32_t snnz = 0;
        scp[0] = 0;
        for (uint32_t j = 0; j < bs; j++) {
            for (uint32_t p = cp[verts[j]]; p < cp[verts[j] + 1]; p++) snnz += blk[ri[p]] == b;
            scp[j + 1] = snnz;
        }
        uint32_t* sri = ws.take(snnz);
        if (!sri && snnz) { ws.used = mark0; return false; }
        for (uint32_t j = 0, w = 0; j < bs; j++)
            for (uint32_t p = cp[verts[j]]; p < cp[verts[j] + 1]; p++)
                if (blk[ri[p]] == b) sri[w++] = loc[ri[p]];
        uint32_t* sq = ws.take(bs);
        if (!sq || !amd_order(bs, scp, sri, sq, ws)) { ws.used = mark0; return false; }
        uint32_t* nat = ws.take(bs);
        if (!nat) { ws.used = mark0; return false; }
        std::memcpy(nat, verts, sizeof(uint32_t) * bs);
        std::sort(nat, nat + bs);
        for (uint32_t i = 0; i < bs; i++) nat[i] = loc[nat[i]];
        uint64_t ac = chol_count(bs, scp, sri, sq, ws, kCountFail);
        if (ac == kCountFail) { ws.used = mark0; return false; }
        uint64_t nc = chol_count(bs, scp, sri, nat, ws, ac);
        if (nc == kCountFail) { ws.used = mark0; return false; }
        const uint32_t* ord = nc < ac ? nat : sq;
        for (uint32_t i = 0; i < bs; i++) q[lo + i] = verts[ord[i]];
        ws.used = bmark;
    }
    ws.used = mark0;
    return true;
}

// ---------------------------------------------------------------------------
// The lead lane's factor.

struct Panel { uint32_t first, last, row_off, val_off; };

inline uint64_t bits(double x) { uint64_t b; std::memcpy(&b, &x, 8); return b; }
inline bool finite(double x) { return std::fabs(x) <= std::numeric_limits<double>::max(); }

struct Factor {
    uint32_t n, nnz;
    const uint32_t *cp, *ri;
    const std::vector<uint32_t>& q;
    std::vector<uint32_t> pinv, lp, up, prow, li, ui, void_slots;
    std::vector<double> lx, ux, udiag, w, y, rscale;
    std::vector<uint8_t> void_col, scaled;
    std::vector<uint32_t> want, want_of, prev, flag, topo, stack, pstack, lend, sn_of, sn_slot, sn_end;
    bool sn_dfs = false;
    std::vector<Panel> panels;
    std::vector<uint32_t> panel_rows;
    std::vector<double> panel_vals;
    double keep_min = kGrowthLimit;

    Factor(uint32_t n_, const uint32_t* cp_, const uint32_t* ri_, const std::vector<uint32_t>& q_)
        : n(n_), nnz(cp_[n_]), cp(cp_), ri(ri_), q(q_) {
        pinv.assign(n, kNone);
        lp.assign(n + 1, 0);
        up.assign(n + 1, 0);
        prow.assign(nnz, 0);
        udiag.assign(n, 0);
        w.assign(n, 0);
        y.assign(n, 0);
        rscale.assign(n, 0);
        void_col.assign(n, 0);
        scaled.assign(n, 0);
        for (auto* v : {&want, &want_of, &prev, &flag, &topo, &stack, &pstack, &lend, &sn_of, &sn_slot, &sn_end})
            v->assign(n, 0);
    }

    uint32_t panel_end(uint32_t kc) const {
        const Panel& pan = panels[sn_of[kc]];
        return pan.row_off + lp[pan.first + 1] - lp[pan.first];
    }

    uint32_t enter(uint32_t r, uint32_t sp, uint32_t mark) {
        uint32_t kc = pinv[r];
        sn_end[sp] = kNone;
        if (kc == kNone) return 0;
        uint32_t id = sn_of[kc];
        if (id == kNone || !sn_dfs) return lp[kc];
        Panel pan = panels[id];
        const uint32_t* rows = panel_rows.data() + pan.row_off;
        uint32_t e = kc;
        while (e < pan.last && flag[rows[e - pan.first]] != mark) { flag[rows[e - pan.first]] = mark; e++; }
        sn_end[sp] = e;
        return e == pan.last ? pan.row_off + (pan.last - pan.first + 1) - 1 : panel_end(kc);
    }

    void grow_panel(uint32_t k, uint32_t piv) {
        if (sn_of[k - 1] == kNone) {
            uint32_t f = k - 1;
            sn_of[f] = uint32_t(panels.size());
            panels.push_back({f, f, uint32_t(panel_rows.size()), uint32_t(panel_vals.size())});
            for (uint32_t p = lp[f], i = 0; p < lp[k]; p++, i++) {
                sn_slot[li[p]] = i;
                panel_rows.push_back(li[p]);
                panel_vals.push_back(lx[p]);
            }
        }
        uint32_t pid = sn_of[k - 1];
        Panel& pan = panels[pid];
        uint32_t nrows = lp[pan.first + 1] - lp[pan.first];
        uint32_t* rows = panel_rows.data() + pan.row_off;
        uint32_t b = k - pan.first - 1, a = sn_slot[piv];
        if (a != b) {
            double* vals = panel_vals.data() + pan.val_off;
            for (uint32_t col = 0; col < k - pan.first; col++) std::swap(vals[col * nrows + a], vals[col * nrows + b]);
            sn_slot[rows[b]] = a;
            sn_slot[piv] = b;
            std::swap(rows[a], rows[b]);
        }
        size_t d0 = panel_vals.size();
        panel_vals.resize(d0 + nrows, 0.0);
        for (size_t p = lp[k]; p < li.size(); p++) panel_vals[d0 + sn_slot[li[p]]] = lx[p];
        pan.last = k;
        sn_of[k] = pid;
    }

    void link_step(uint32_t k, uint32_t piv, uint32_t mark) {
        uint32_t s = k - 1, at = kNone, last_out = kNone;
        for (uint32_t p = lp[s], i = 0; p < lp[k]; p++, i++) {
            uint32_t r = li[p];
            if (r == piv) at = i;
            else if (flag[r] != mark || pinv[r] != kNone) last_out = i;
        }
        if (at == kNone || (last_out != kNone && last_out > at)) return;
        lend[s] = lp[s] + at + 1;
        if (last_out == kNone && lp[k] - lp[s] == li.size() - lp[k] + 1) grow_panel(k, piv);
    }

    uint32_t panel_run(uint32_t idx0, uint32_t kc) {
        Panel pan = panels[sn_of[kc]];
        uint32_t nrows = lp[pan.first + 1] - lp[pan.first], m = pan.last - pan.first + 1;
        const uint32_t* rows = panel_rows.data() + pan.row_off;
        const double* vals = panel_vals.data() + pan.val_off;
        uint32_t len = 1;
        while (kc + len <= pan.last && len <= idx0 && pinv[topo[idx0 - len]] == kc + len) len++;
        uint32_t b0 = kc - pan.first, xn = m - 1 - b0;
        double* x = y.data();
        for (uint32_t i = 0; i < xn; i++) x[i] = w[rows[b0 + i]];
        size_t run0 = ux.size();
        for (uint32_t j = 0; j < len; j++) {
            uint32_t t = kc + j;
            double ut = j == 0 ? w[topo[idx0]] : x[j - 1];
            ui.push_back(t);
            ux.push_back(ut);
            const double* col = vals + size_t(t - pan.first) * nrows;
            for (uint32_t i = j; i < xn; i++) x[i] -= col[b0 + i] * ut;
        }
        for (uint32_t i = 0; i < xn; i++) w[rows[b0 + i]] = x[i];
        const double* cv = vals + size_t(b0) * nrows;
        for (uint32_t i = m - 1; i < nrows; i++) {
            double acc = w[rows[i]];
            for (uint32_t j = 0; j < len; j++) acc -= cv[size_t(j) * nrows + i] * ux[run0 + j];
            w[rows[i]] = acc;
        }
        return idx0 - (len - 1);
    }

    bool void_unknown(const double* vals, uint32_t c) const {
        if (pinv[c] != kNone) return false;
        for (uint32_t p = cp[c]; p < cp[c + 1]; p++)
            if (vals[p] != 0) return false;
        for (uint32_t j = 0; j < n; j++) {
            if (j == c) continue;
            for (uint32_t p = cp[j]; p < cp[j + 1]; p++)
                if (ri[p] == c && vals[p] != 0) return false;
        }
        return true;
    }

    // 0 factored, 1 over the cap, -1 singular.
    int pass(const double* vals, size_t cap, bool keep_prev) {
        std::fill(pinv.begin(), pinv.end(), kNone);
        std::fill(flag.begin(), flag.end(), 0);
        std::fill(void_col.begin(), void_col.end(), 0);
        std::fill(scaled.begin(), scaled.end(), 0);
        panels.clear();
        panel_rows.clear();
        panel_vals.clear();
        void_slots.clear();
        li.clear(); lx.clear(); ui.clear(); ux.clear();
        bool has_void = false;
        uint64_t mb = 0;
        for (uint32_t p = 0; p < nnz; p++) mb = std::max(mb, bits(std::fabs(vals[p])));
        double mx; std::memcpy(&mx, &mb, 8);
        if (!(mx <= std::numeric_limits<double>::max())) return -1;
        std::fill(rscale.begin(), rscale.end(), 0.0);
        for (uint32_t j = 0; j < n; j++)
            for (uint32_t p = cp[j]; p < cp[j + 1]; p++) rscale[ri[p]] = std::max(rscale[ri[p]], std::fabs(vals[p]));
        for (auto& s : rscale) s = (s > 0 && finite(s)) ? 1 / s : 1;
        uint64_t nonfinite = 0;
        for (uint32_t i = 0; i < n; i++) want[i] = keep_prev ? prev[i] : i;
        for (uint32_t c = 0; c < n; c++) want_of[want[c]] = c;
        uint32_t k = 0;
        for (int sn = 0; sn <= 1; sn++) {
            if (sn) {
                lp[k] = uint32_t(li.size());
                for (uint32_t t = 0; t < k; t++) lend[t] = lp[t + 1];
                std::fill(sn_of.begin(), sn_of.end(), kNone);
                sn_dfs = false;
            }
            while (k < n) {
                uint32_t c = q[k];
                lp[k] = uint32_t(li.size());
                up[k] = uint32_t(ui.size());
                uint32_t mark = k + 1, nt = 0;
                for (uint32_t p = cp[c]; p < cp[c + 1]; p++) {
                    uint32_t r = ri[p];
                    if (flag[r] == mark) continue;
                    uint32_t sp = 0;
                    stack[0] = r;
                    flag[r] = mark;
                    pstack[0] = sn ? enter(r, 0, mark) : (pinv[r] == kNone ? 0 : lp[pinv[r]]);
                    for (;;) {
                        r = stack[sp];
                        uint32_t kc = pinv[r];
                        bool in_panel = sn && kc != kNone && sn_end[sp] != kNone;
                        const uint32_t* adj = in_panel ? panel_rows.data() : li.data();
                        uint32_t end = kc == kNone ? 0 : in_panel ? panel_end(kc) : sn ? lend[kc] : lp[kc + 1];
                        uint32_t pos = pstack[sp];
                        bool down = false;
                        while (pos < end) {
                            uint32_t ch = adj[pos++];
                            if (flag[ch] != mark) {
                                pstack[sp] = pos;
                                flag[ch] = mark;
                                stack[++sp] = ch;
                                pstack[sp] = sn ? enter(ch, sp, mark) : (pinv[ch] == kNone ? 0 : lp[pinv[ch]]);
                                down = true;
                                break;
                            }
                        }
                        if (down) continue;
                        if (in_panel) {
                            const Panel& pan = panels[sn_of[kc]];
                            const uint32_t* rows = panel_rows.data() + pan.row_off;
                            for (uint32_t t = sn_end[sp]; t > kc; t--) topo[nt++] = rows[t - pan.first - 1];
                        }
                        topo[nt++] = r;
                        if (sp == 0) break;
                        sp--;
                    }
                }
                for (uint32_t p = cp[c]; p < cp[c + 1]; p++) w[ri[p]] = vals[p];
                for (uint32_t idx = nt; idx > 0;) {
                    idx--;
                    uint32_t r = topo[idx], kc = pinv[r];
                    if (kc == kNone) continue;
                    if (sn && !panels.empty() && sn_of[kc] != kNone) { idx = panel_run(idx, kc); continue; }
                    double u = w[r];
                    ui.push_back(kc);
                    ux.push_back(u);
                    for (uint32_t q2 = lp[kc]; q2 < lp[kc + 1]; q2++) w[li[q2]] -= lx[q2] * u;
                }
                double amax = 0, smax = 0;
                uint32_t piv = kNone;
                for (uint32_t t = 0; t < nt; t++) {
                    uint32_t r = topo[t];
                    if (pinv[r] != kNone) continue;
                    double a = std::fabs(w[r]);
                    if (a > amax) { amax = a; piv = r; }
                    double sa = a * rscale[r];
                    smax = (std::isnan(sa) || std::isnan(smax)) ? NAN : std::max(smax, sa);
                }
                if (piv == kNone || amax == 0 || !finite(amax)) {
                    if (!void_unknown(vals, c)) {
                        for (uint32_t t = 0; t < nt; t++) w[topo[t]] = 0;
                        return -1;
                    }
                    void_col[k] = 1;
                    has_void = true;
                    udiag[k] = 1;
                    pinv[c] = k;
                    if (sn) lend[k] = lp[k];
                    for (uint32_t t = 0; t < nt; t++) w[topo[t]] = 0;
                    k++;
                    continue;
                }
                uint32_t pr = want[c];
                if (pinv[pr] == kNone) {
                    double dmag = std::fabs(w[pr]);
                    if (keep_prev) {
                        if (dmag > 0 && dmag >= keep_min * amax) piv = pr;
                    } else if (dmag > 0 && dmag >= kPivotTol * amax) {
                        piv = pr;
                    } else if (dmag > 0 && dmag * rscale[pr] >= kPivotTol * smax) {
                        piv = pr;
                        scaled[k] = 1;
                    }
                }
                if (piv != pr) {
                    uint32_t c2 = want_of[piv];
                    want[c2] = pr;
                    want_of[pr] = c2;
                }
                double d = w[piv];
                udiag[k] = d;
                pinv[piv] = k;
                for (uint32_t t = 0; t < nt; t++) {
                    uint32_t r = topo[t];
                    double v = w[r];
                    nonfinite |= bits(v - v);
                    if (pinv[r] == kNone) {
                        double l = v / d;
                        nonfinite |= bits(l - l);
                        li.push_back(r);
                        lx.push_back(l);
                    }
                    w[r] = 0;
                }
                if (li.size() + ui.size() > cap) return 1;
                if (!sn) {
                    bool out = li.size() - lp[k] >= 32;
                    k++;
                    if (out) break;
                    continue;
                }
                lend[k] = uint32_t(li.size());
                if (k > 0 && (lp[k] - lp[k - 1] >= 32 || sn_of[k - 1] != kNone)) link_step(k, piv, mark);
                if (panel_vals.size() >= li.size() / 5 * 4) sn_dfs = true;
                k++;
            }
        }
        lp[n] = uint32_t(li.size());
        up[n] = uint32_t(ui.size());
        if (nonfinite) return -1;
        for (auto& r : li) r = pinv[r];
        for (uint32_t p = 0; p < nnz; p++) prow[p] = pinv[ri[p]];
        if (has_void)
            for (uint32_t j = 0; j < n; j++)
                for (uint32_t p = cp[q[j]]; p < cp[q[j] + 1]; p++)
                    if (void_col[j] || void_col[prow[p]]) void_slots.push_back(p);
        return 0;
    }
};

}  // namespace

bool order_columns(uint32_t n, const uint32_t* col_ptr, const uint32_t* row_idx, std::vector<uint32_t>& q) {
    q.assign(n, 0);
    Slab ws(slab_words(n, col_ptr[n]));
    return order_in(n, col_ptr, row_idx, q.data(), ws);
}

uint64_t diag_fill(uint32_t n, const uint32_t* col_ptr, const uint32_t* row_idx, const std::vector<uint32_t>& q) {
    Slab ws(slab_words(n, col_ptr[n]));
    uint64_t c = chol_count(n, col_ptr, row_idx, q.data(), ws, kCountFail);
    return 2 * (c - n);
}

bool factor_tape(uint32_t n, const uint32_t* col_ptr, const uint32_t* row_idx, const double* vals,
                 const std::vector<uint32_t>& q, Tape& out) {
    Factor f(n, col_ptr, row_idx, q);
    // A first factor with the solver's fill cap (direct.zig:232-245 with
    // sparse_lu.zig:295-298): past 3 x diag_fill it restarts on the diagonal.
    uint64_t df = std::max<uint64_t>(diag_fill(n, col_ptr, row_idx, q), col_ptr[n]);
    double c = kRepivotFillCap * double(df);
    size_t cap = size_t(c < 1e18 ? c : 1e18);
    for (uint32_t i = 0; i < n; i++) f.prev[i] = i;
    int r = f.pass(vals, cap, false);
    if (r < 0) return false;
    if (r == 1 && f.pass(vals, cap, true) != 0) return false;
    out.n = n;
    out.nnz = col_ptr[n];
    out.q = q;
    out.pinv = f.pinv;
    out.lp = f.lp;
    out.up = f.up;
    out.li = f.li;
    out.ui = f.ui;
    out.prow = f.prow;
    out.void_slots = f.void_slots;
    out.flags.assign(n, 0);
    for (uint32_t k = 0; k < n; k++) out.flags[k] = (f.void_col[k] ? kVoidBit : 0) | (f.scaled[k] ? kScaledBit : 0);
    out.lx = f.lx;
    out.ux = f.ux;
    out.udiag = f.udiag;
    out.sn_dfs = f.sn_dfs;
    out.panels = uint32_t(f.panels.size());
    return true;
}

bool lu_program(const Tape& t, const uint32_t* col_ptr, std::vector<uint32_t>& prog) {
    prog.clear();
    const uint32_t n = t.n;
    auto fits = [](uint64_t v) { return v < 65536u; };
    if (!fits(n) || !fits(t.prow.size()) || !fits(t.li.size()) || !fits(t.ui.size())) return false;
    auto pack = [](uint32_t hi, uint32_t lo) { return (hi << 16) | lo; };
    for (uint32_t k = 0; k < n; k++) {
        uint32_t c = t.q[k];
        uint32_t fl = t.flags[k];
        uint32_t cnt = col_ptr[c + 1] - col_ptr[c];
        if (cnt) {
            prog.push_back(kOpScat | (cnt << 4));
            for (uint32_t p = col_ptr[c]; p < col_ptr[c + 1]; p++) prog.push_back(pack(t.prow[p], p));
        }
        for (uint32_t p = t.up[k]; p < t.up[k + 1]; p++) {
            uint32_t i = t.ui[p];
            uint32_t m = t.lp[i + 1] - t.lp[i];
            prog.push_back(kOpTake | (m << 4));
            prog.push_back(pack(i, p));
            for (uint32_t pl = t.lp[i]; pl < t.lp[i + 1]; pl++) prog.push_back(pack(t.li[pl], pl));
        }
        if (fl & 1u) {
            prog.push_back(kOpVoid);
            prog.push_back(k);
            continue;
        }
        uint32_t m = t.lp[k + 1] - t.lp[k];
        prog.push_back(kOpPiv | ((fl & 15u) << 4) | (m << 8));
        prog.push_back(k);
        for (uint32_t p = t.lp[k]; p < t.lp[k + 1]; p++) prog.push_back(pack(t.li[p], p));
    }
    prog.push_back(kOpEnd);
    return true;
}

bool lu_records(const Tape& t, const uint32_t* col_ptr, std::vector<uint32_t>& rec) {
    rec.clear();
    const uint32_t n = t.n;
    auto fits = [](uint64_t v) { return v < 65536u; };
    if (!fits(n) || !fits(t.prow.size()) || !fits(t.li.size()) || !fits(t.ui.size())) return false;
    auto pack = [](uint32_t hi, uint32_t lo) { return (hi << 16) | lo; };
    auto put = [&](uint32_t x, uint32_t y, uint32_t z, uint32_t w) {
        rec.push_back(x);
        rec.push_back(y);
        rec.push_back(z);
        rec.push_back(w);
    };
    std::vector<uint32_t> e;
    for (uint32_t k = 0; k < n; k++) {
        const uint32_t c = t.q[k];
        const uint32_t fl = t.flags[k];
        e.clear();
        for (uint32_t p = col_ptr[c]; p < col_ptr[c + 1]; p++) e.push_back(pack(t.prow[p], p));
        for (size_t j = 0; j < e.size(); j += 3) {
            const uint32_t m = (uint32_t)std::min<size_t>(3, e.size() - j);
            put(kRecScat | (m << 4), e[j], m > 1 ? e[j + 1] : 0u, m > 2 ? e[j + 2] : 0u);
        }
        for (uint32_t p = t.up[k]; p < t.up[k + 1]; p++) {
            const uint32_t i = t.ui[p];
            e.clear();
            for (uint32_t pl = t.lp[i]; pl < t.lp[i + 1]; pl++) e.push_back(pack(t.li[pl], pl));
            const uint32_t m0 = (uint32_t)std::min<size_t>(2, e.size());
            put(kRecTake | (m0 << 4) | (i << 16), p, m0 > 0 ? e[0] : 0u, m0 > 1 ? e[1] : 0u);
            for (size_t j = m0; j < e.size(); j += 3) {
                const uint32_t m = (uint32_t)std::min<size_t>(3, e.size() - j);
                put(kRecAxpy | (m << 4), e[j], m > 1 ? e[j + 1] : 0u, m > 2 ? e[j + 2] : 0u);
            }
        }
        if (fl & 1u) {
            put(kRecVoid | (k << 16), 0, 0, 0);
            continue;
        }
        e.clear();
        for (uint32_t p = t.lp[k]; p < t.lp[k + 1]; p++) e.push_back(pack(t.li[p], p));
        const uint32_t m0 = (uint32_t)std::min<size_t>(3, e.size());
        const uint32_t last0 = e.size() <= 3 ? 1u : 0u;
        put(kRecPiv | (m0 << 4) | ((fl & 15u) << 8) | (last0 << 12) | (k << 16), m0 > 0 ? e[0] : 0u,
            m0 > 1 ? e[1] : 0u, m0 > 2 ? e[2] : 0u);
        for (size_t j = m0; j < e.size(); j += 3) {
            const uint32_t m = (uint32_t)std::min<size_t>(3, e.size() - j);
            const uint32_t last = j + m == e.size() ? 1u : 0u;
            put(kRecDiv | (m << 4) | (last << 12), e[j], m > 1 ? e[j + 1] : 0u, m > 2 ? e[j + 2] : 0u);
        }
    }
    put(kRecEnd, 0, 0, 0);
    put(kRecEnd, 0, 0, 0);
    return true;
}

bool solve_records(const Tape& t, std::vector<uint32_t>& rec) {
    rec.clear();
    const uint32_t n = t.n;
    auto fits = [](uint64_t v) { return v < 65536u; };
    if (!fits(n) || !fits(t.li.size()) || !fits(t.ui.size())) return false;
    auto put = [&](uint32_t x, uint32_t y, uint32_t z, uint32_t w) {
        rec.push_back(x);
        rec.push_back(y);
        rec.push_back(z);
        rec.push_back(w);
    };
    std::vector<uint32_t> e;
    auto column = [&](uint32_t first, uint32_t cont, uint32_t k, bool always) {
        if (e.empty() && !always) return;
        const uint32_t m0 = (uint32_t)std::min<size_t>(3, e.size());
        put(first | (m0 << 4) | (k << 16), m0 > 0 ? e[0] : 0u, m0 > 1 ? e[1] : 0u, m0 > 2 ? e[2] : 0u);
        for (size_t j = m0; j < e.size(); j += 3) {
            const uint32_t m = (uint32_t)std::min<size_t>(3, e.size() - j);
            put(cont | (m << 4), e[j], m > 1 ? e[j + 1] : 0u, m > 2 ? e[j + 2] : 0u);
        }
    };
    for (uint32_t k = 0; k < n; k++) {
        e.clear();
        for (uint32_t p = t.lp[k]; p < t.lp[k + 1]; p++) e.push_back((t.li[p] << 16) | p);
        column(kSolFwd, kSolFwdC, k, false);
    }
    for (uint32_t k = n; k-- > 0;) {
        e.clear();
        for (uint32_t p = t.up[k]; p < t.up[k + 1]; p++) e.push_back((t.ui[p] << 16) | p);
        column(kSolBwd, kSolBwdC, k, true);
    }
    put(kSolEnd, 0, 0, 0);
    put(kSolEnd, 0, 0, 0);
    return true;
}

namespace {
uint32_t pow2_at_least(uint32_t v) {
    uint32_t p = 1;
    while (p < v) p <<= 1;
    return p;
}
}  // namespace

bool band_plan(const Tape& t, const std::vector<uint32_t>& prog, uint32_t max_band, uint32_t max_l_ring,
               uint32_t chunk_words, uint32_t chunk_entries, BandPlan& out) {
    out = BandPlan{};
    const uint32_t n = t.n;
    if (prog.empty() || n == 0) return false;
    for (uint32_t k = 0; k < n; k++)
        if (t.flags[k] & 1u) return false;
    // the band: every row the replay and the solves touch at column k
    uint32_t band = 0;
    auto see = [&](uint32_t r, uint32_t k) { band = std::max(band, r > k ? r - k : k - r); };
    {
        uint32_t k = 0;
        for (uint32_t pc = 0; pc < prog.size();) {
            uint32_t h = prog[pc], op = h & 15u;
            if (op == kOpEnd) break;
            if (op == kOpScat) {
                uint32_t cnt = h >> 4;
                for (uint32_t j = 0; j < cnt; j++) see(prog[pc + 1 + j] >> 16, k);
                pc += 1 + cnt;
            } else if (op == kOpTake) {
                uint32_t cnt = h >> 4;
                see(prog[pc + 1] >> 16, k);
                for (uint32_t j = 0; j < cnt; j++) see(prog[pc + 2 + j] >> 16, k);
                pc += 2 + cnt;
            } else if (op == kOpPiv) {
                uint32_t cnt = h >> 8;
                k = prog[pc + 1];
                see(k, k);
                for (uint32_t j = 0; j < cnt; j++) see(prog[pc + 2 + j] >> 16, k);
                pc += 2 + cnt;
                k++;
            } else {
                return false;
            }
        }
    }
    // (a column's scatter and take entries come before its pivot op, which
    // names k; the running k is already that column)
    if (band > max_band) return false;
    uint32_t lwin = 0;
    for (uint32_t k = 0; k < n; k++) {
        uint32_t k0 = k > band ? k - band : 0;
        lwin = std::max(lwin, t.lp[k + 1] - t.lp[k0]);
    }
    out.band = band;
    out.w_ring = pow2_at_least(2 * band + 2);
    out.l_ring = pow2_at_least(std::max(lwin, 1u));
    if (out.l_ring > max_l_ring) return false;
    // chunks on op boundaries
    uint32_t words = 0, entries = 0, e = 0;
    out.chunk_pc.push_back(0);
    out.chunk_e.push_back(0);
    for (uint32_t pc = 0; pc < prog.size();) {
        uint32_t h = prog[pc], op = h & 15u;
        uint32_t size = 1, ents = 0;
        if (op == kOpEnd) break;
        if (op == kOpScat) {
            size = 1 + (h >> 4);
            ents = h >> 4;
            for (uint32_t j = 0; j < ents; j++) out.scat_slot.push_back(prog[pc + 1 + j] & 0xffffu);
        } else if (op == kOpTake) {
            size = 2 + (h >> 4);
        } else {
            size = 2 + (h >> 8);
        }
        if (size > chunk_words || ents > chunk_entries) return false;
        if (words + size > chunk_words || entries + ents > chunk_entries) {
            out.chunk_pc.push_back(pc);
            out.chunk_e.push_back(e);
            words = entries = 0;
        }
        words += size;
        entries += ents;
        e += ents;
        pc += size;
    }
    uint32_t end = 0;
    while (end < prog.size() && prog[end] != kOpEnd) {
        uint32_t h = prog[end], op = h & 15u;
        end += op == kOpScat ? 1 + (h >> 4) : op == kOpTake ? 2 + (h >> 4) : 2 + (h >> 8);
    }
    out.chunk_pc.push_back(end);
    out.chunk_e.push_back(e);
    out.max_words = chunk_words;
    out.max_entries = chunk_entries;
    // column blocks of the solves
    out.solve_col.push_back(0);
    uint32_t k0 = 0;
    for (uint32_t k = 0; k < n; k++) {
        uint32_t nl = t.lp[k + 1] - t.lp[k0], nu = t.up[k + 1] - t.up[k0];
        if (t.lp[k + 1] - t.lp[k] > kSolveEntries || t.up[k + 1] - t.up[k] > kSolveEntries) return false;
        if (k + 1 - k0 > kSolveCols || nl > kSolveEntries || nu > kSolveEntries) {
            out.solve_col.push_back(k);
            k0 = k;
        }
    }
    out.solve_col.push_back(n);
    out.rowof.assign(n, 0);
    for (uint32_t r = 0; r < n; r++) out.rowof[t.pinv[r]] = r;
    return true;
}

void level_plan(const Tape& t, LevelPlan& out) {
    const uint32_t n = t.n;
    // rows of L: column k's entries (row li[p] > k, slot p) go to row li[p]
    auto by_rows = [n](const std::vector<uint32_t>& cptr, const std::vector<uint32_t>& rows,
                       std::vector<uint32_t>& rptr, std::vector<uint32_t>& ent) {
        rptr.assign(n + 1, 0);
        for (uint32_t r : rows) rptr[r + 1]++;
        for (uint32_t i = 0; i < n; i++) rptr[i + 1] += rptr[i];
        ent.assign(2 * (size_t)rows.size(), 0);
        std::vector<uint32_t> fill(rptr.begin(), rptr.end() - 1);
        for (uint32_t k = 0; k < n; k++)
            for (uint32_t p = cptr[k]; p < cptr[k + 1]; p++) {
                const uint32_t e = fill[rows[p]]++;
                ent[2 * (size_t)e] = k;
                ent[2 * (size_t)e + 1] = p;
            }
    };
    by_rows(t.lp, t.li, out.rl_ptr, out.rl_ent);
    by_rows(t.up, t.ui, out.ru_ptr, out.ru_ent);
    auto bucket = [n](const std::vector<uint32_t>& lev, std::vector<uint32_t>& ptr, std::vector<uint32_t>& rows) {
        uint32_t top = 0;
        for (uint32_t v : lev) top = std::max(top, v + 1);
        ptr.assign(top + 1, 0);
        for (uint32_t v : lev) ptr[v + 1]++;
        for (uint32_t v = 0; v < top; v++) ptr[v + 1] += ptr[v];
        rows.assign(n, 0);
        std::vector<uint32_t> fill(ptr.begin(), ptr.end() - 1);
        for (uint32_t i = 0; i < n; i++) rows[fill[lev[i]]++] = i;
    };
    std::vector<uint32_t> lev(n, 0);
    for (uint32_t i = 0; i < n; i++) {
        uint32_t v = 0;
        for (uint32_t e = out.rl_ptr[i]; e < out.rl_ptr[i + 1]; e++) v = std::max(v, lev[out.rl_ent[2 * (size_t)e]] + 1);
        lev[i] = v;
    }
    bucket(lev, out.fl_ptr, out.fl_rows);
    for (uint32_t j = n; j-- > 0;) {
        uint32_t v = 0;
        for (uint32_t e = out.ru_ptr[j]; e < out.ru_ptr[j + 1]; e++) v = std::max(v, lev[out.ru_ent[2 * (size_t)e]] + 1);
        lev[j] = v;
    }
    bucket(lev, out.bl_ptr, out.bl_rows);
}

void col_plan(const Tape& t, uint32_t max_groups, ColPlan& out) {
    out = ColPlan{};
    const uint32_t n = t.n;
    std::vector<uint32_t> lev(n, 0);
    std::vector<uint64_t> work(n, 0);
    uint32_t top = 0;
    for (uint32_t k = 0; k < n; k++) {
        uint32_t v = 0;
        uint64_t wk = 1 + (t.lp[k + 1] - t.lp[k]);
        for (uint32_t p = t.up[k]; p < t.up[k + 1]; p++) {
            const uint32_t i = t.ui[p];
            v = std::max(v, lev[i] + 1);
            wk += 1 + (t.lp[i + 1] - t.lp[i]);
        }
        lev[k] = v;
        work[k] = wk;
        top = std::max(top, v + 1);
    }
    out.ustream.resize(4 * (size_t)t.ui.size());
    for (size_t p = 0; p < t.ui.size(); p++) {
        const uint32_t i = t.ui[p];
        out.ustream[4 * p] = i;
        out.ustream[4 * p + 1] = t.lp[i];
        out.ustream[4 * p + 2] = t.lp[i + 1];
        out.ustream[4 * p + 3] = 0;
    }
    std::vector<std::vector<uint32_t>> by(top);
    for (uint32_t k = 0; k < n; k++) by[lev[k]].push_back(k);
    out.lv_ptr.push_back(0);
    for (uint32_t v = 0; v < top; v++) {
        const auto& cs = by[v];
        uint32_t G = 1;
        while (G * 2 <= std::min<uint32_t>(max_groups, (uint32_t)cs.size())) G *= 2;
        // the heaviest columns first, each to the least loaded group
        std::vector<uint32_t> order(cs.begin(), cs.end());
        std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return work[a] > work[b]; });
        std::vector<uint64_t> load(G, 0);
        std::vector<std::vector<uint32_t>> grp(G);
        for (uint32_t k : order) {
            const uint32_t g = (uint32_t)(std::min_element(load.begin(), load.end()) - load.begin());
            grp[g].push_back(k);
            load[g] += work[k];
        }
        for (uint32_t g = 0; g < G; g++) {
            std::sort(grp[g].begin(), grp[g].end());
            out.gp.push_back((uint32_t)out.cols.size());
            out.cols.insert(out.cols.end(), grp[g].begin(), grp[g].end());
        }
        out.gp.push_back((uint32_t)out.cols.size());
        out.lv_ptr.push_back((uint32_t)out.gp.size());
    }
}

bool stream_plan(const std::vector<uint32_t>& lev_ptr, const std::vector<uint32_t>& rows,
                 const std::vector<uint32_t>& row_ptr, const std::vector<uint32_t>& ent, uint32_t chunk,
                 uint32_t max_rows, uint32_t ahead, bool skip_empty, StreamPlan& out) {
    out = StreamPlan{};
    out.ch.push_back(0);
    out.mo.push_back(0);
    // the open chunk: its segments (3 words each), rows and entry offsets
    std::vector<uint32_t> seg, ri, rp;
    // the chunk and position that compute each row
    const size_t n = row_ptr.empty() ? 0 : row_ptr.size() - 1;
    std::vector<uint32_t> in_chunk(n, kNone), at(n, 0);
    uint32_t e = 0, c0 = 0;  // next entry, first entry of the open chunk
    auto close = [&]() {
        if (ri.empty()) return;
        while (e % 4u) {  // the next chunk starts on a multiple of four entries
            out.col.push_back(0);
            out.slot.push_back(kNone);
            e++;
        }
        rp.push_back(e - c0);
        const uint32_t ns = (uint32_t)seg.size() / 3, nr = (uint32_t)ri.size();
        const size_t m0 = out.meta.size();
        out.meta.insert(out.meta.end(), {ns, nr, e - c0, 0u, 0u, 0u, 0u, 0u});
        out.meta.insert(out.meta.end(), seg.begin(), seg.end());
        out.meta.insert(out.meta.end(), ri.begin(), ri.end());
        out.meta.insert(out.meta.end(), rp.begin(), rp.end());
        while (out.meta.size() % 4u) out.meta.push_back(0);
        out.max_meta = std::max(out.max_meta, (uint32_t)(out.meta.size() - m0));
        out.ch.push_back(e);
        out.mo.push_back((uint32_t)out.meta.size());
        seg.clear();
        ri.clear();
        rp.clear();
        c0 = e;
    };
    for (size_t v = 0; v + 1 < lev_ptr.size(); v++) {
        bool open = false;  // a segment of this level is open in the chunk
        for (uint32_t k = lev_ptr[v]; k < lev_ptr[v + 1]; k++) {
            const uint32_t i = rows[k];
            const uint32_t len = row_ptr[i + 1] - row_ptr[i];
            if (len > chunk) return false;
            if (len == 0 && skip_empty) continue;
            if (e - c0 + len > chunk || ri.size() + 1 > max_rows) {
                close();
                open = false;
            }
            if (!open) {
                seg.insert(seg.end(), {(uint32_t)ri.size(), (uint32_t)ri.size(), 0u});
                open = true;
            }
            const uint32_t cur = (uint32_t)out.ch.size() - 1;
            in_chunk[i] = cur;
            at[i] = (uint32_t)ri.size();
            ri.push_back(i);
            rp.push_back(e - c0);
            seg.back() = std::max(seg.back(), len << 1);
            for (uint32_t p = row_ptr[i]; p < row_ptr[i + 1]; p++) {
                const uint32_t j = ent[2 * (size_t)p];
                out.col.push_back(in_chunk[j] == cur ? (kStreamLocal | at[j]) : j);
                out.slot.push_back(ent[2 * (size_t)p + 1]);
                e++;
            }
            seg[seg.size() - 2] = (uint32_t)ri.size();
        }
        if (open) seg.back() |= 1u;  // the level's last segment
    }
    close();
    out.entries = e;
    out.n_chunks = (uint32_t)out.ch.size() - 1;
    for (uint32_t c = 0; c + ahead < out.n_chunks; c++) {
        const uint32_t a = c + ahead;
        uint32_t* h = out.meta.data() + out.mo[c];
        h[4] = out.ch[a];
        h[5] = out.ch[a + 1] - out.ch[a];
        h[6] = out.mo[a];
        h[7] = out.mo[a + 1] - out.mo[a];
    }
    return true;
}

}  // namespace espl
