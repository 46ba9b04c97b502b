// Host check of the large-template LU plans (tape.h): the streaming plan of
// each solve sweep and the refactor's column plan, built from a real factor
// of the CSC matrix given on the command line. Exit status 0 when every
// invariant the kernels rely on holds.
//   plans_host col_ptr.bin row_idx.bin vals.bin q.bin chunk rows ahead groups
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "tape.h"

using namespace espl;

static std::vector<uint8_t> slurp(const char* f) {
    std::vector<uint8_t> v;
    FILE* p = std::fopen(f, "rb");
    if (!p) return v;
    int c;
    while ((c = std::fgetc(p)) != EOF) v.push_back((uint8_t)c);
    std::fclose(p);
    return v;
}
template <class T>
static std::vector<T> as(const std::vector<uint8_t>& b) {
    std::vector<T> v(b.size() / sizeof(T));
    std::memcpy(v.data(), b.data(), v.size() * sizeof(T));
    return v;
}

static int fails = 0;
#define CHECK(cond, ...)                  \
    do {                                  \
        if (!(cond)) {                    \
            std::printf(__VA_ARGS__);     \
            std::printf("\n");            \
            if (++fails > 20) std::exit(1); \
        }                                 \
    } while (0)

// The streaming plan of one sweep: chunk shapes and alignment, each chunk's
// plan, rows in level order with their entries, local columns, level ends.
static void check_stream(const char* name, const std::vector<uint32_t>& lev_ptr, const std::vector<uint32_t>& rows,
                         const std::vector<uint32_t>& row_ptr, const std::vector<uint32_t>& ent, bool skip,
                         uint32_t chunk, uint32_t max_rows, uint32_t ahead) {
    StreamPlan sp;
    CHECK(stream_plan(lev_ptr, rows, row_ptr, ent, chunk, max_rows, ahead, skip, sp), "%s: no plan", name);
    const uint32_t meta_words = (8 + 5 * max_rows + 1 + 3) & ~3u;
    CHECK(sp.max_meta <= meta_words, "%s: plan of %u words", name, sp.max_meta);
    CHECK(sp.entries % 4 == 0 && sp.col.size() == sp.entries && sp.slot.size() == sp.entries, "%s: entries", name);
    std::vector<uint32_t> seen;
    size_t level_ends = 0;
    for (uint32_t c = 0; c < sp.n_chunks; c++) {
        const uint32_t e0 = sp.ch[c], len = sp.ch[c + 1] - e0, m0 = sp.mo[c], ml = sp.mo[c + 1] - m0;
        CHECK(e0 % 4 == 0 && len % 4 == 0 && len && len <= chunk && m0 % 4 == 0 && ml % 4 == 0 && ml <= meta_words,
              "%s: chunk %u shape", name, c);
        const uint32_t* m = sp.meta.data() + m0;
        const uint32_t ns = m[0], nr = m[1];
        CHECK(m[2] == len && nr <= max_rows && ns <= nr && 8 + 3 * ns + 2 * nr + 1 <= ml, "%s: chunk %u header", name,
              c);
        if (c + ahead < sp.n_chunks) {
            const uint32_t a = c + ahead;
            CHECK(m[4] == sp.ch[a] && m[5] == sp.ch[a + 1] - sp.ch[a] && m[6] == sp.mo[a] &&
                      m[7] == sp.mo[a + 1] - sp.mo[a],
                  "%s: chunk %u copy header", name, c);
        }
        const uint32_t *sg = m + 8, *ri = sg + 3 * ns, *rp = ri + nr;
        uint32_t next = 0;
        for (uint32_t g = 0; g < ns; g++) {
            const uint32_t k0 = sg[3 * g], k1 = sg[3 * g + 1], longest = sg[3 * g + 2] >> 1;
            level_ends += sg[3 * g + 2] & 1u;
            CHECK(k0 == next && k0 < k1 && k1 <= nr, "%s: chunk %u segment %u", name, c, g);
            next = k1;
            uint32_t mx = 0;
            for (uint32_t k = k0; k < k1; k++) {
                const uint32_t i = ri[k], n_real = row_ptr[i + 1] - row_ptr[i];
                mx = std::max(mx, n_real);
                seen.push_back(i);
                CHECK(rp[k] <= rp[k + 1] && rp[k + 1] <= len && rp[k + 1] - rp[k] >= n_real, "%s: row %u offsets",
                      name, i);
                for (uint32_t t = 0; t < n_real; t++) {
                    const uint32_t e = e0 + rp[k] + t, p = row_ptr[i] + t, code = sp.col[e];
                    const bool col_ok = (code & kStreamLocal)
                                            ? ((code & ~kStreamLocal) < k && ri[code & ~kStreamLocal] == ent[2 * p])
                                            : code == ent[2 * p];
                    CHECK(col_ok && sp.slot[e] == ent[2 * p + 1], "%s: row %u entry %u", name, i, t);
                }
                for (uint32_t e = e0 + rp[k] + n_real; e < e0 + rp[k + 1]; e++)
                    CHECK(sp.slot[e] == kNone, "%s: padding of row %u", name, i);
            }
            CHECK(mx == longest, "%s: chunk %u segment %u longest row", name, c, g);
        }
        CHECK(next == nr, "%s: chunk %u rows", name, c);
    }
    std::vector<uint32_t> want;
    size_t levels = 0;
    for (size_t v = 0; v + 1 < lev_ptr.size(); v++) {
        bool any = false;
        for (uint32_t k = lev_ptr[v]; k < lev_ptr[v + 1]; k++) {
            const uint32_t i = rows[k];
            if (skip && row_ptr[i + 1] == row_ptr[i]) continue;
            want.push_back(i);
            any = true;
        }
        levels += any ? 1 : 0;
    }
    CHECK(want == seen, "%s: rows not in level order", name);
    CHECK(level_ends == levels, "%s: %zu level ends for %zu levels", name, level_ends, levels);
    std::printf("%s: %u chunks, %u entries, %zu levels\n", name, sp.n_chunks, sp.entries, levels);
}

// The refactor's column plan: every column once, a level's columns reading
// only earlier levels, groups a power of two no more than the level's
// columns or the cap, the entry stream.
static void check_columns(const Tape& t, uint32_t groups) {
    ColPlan cp;
    col_plan(t, groups, cp);
    const uint32_t n = t.n;
    std::vector<int> level(n, -1);
    size_t count = 0;
    for (size_t v = 0; v + 1 < cp.lv_ptr.size(); v++) {
        const uint32_t b = cp.lv_ptr[v], G = cp.lv_ptr[v + 1] - b - 1;
        CHECK(G >= 1 && G <= groups && (G & (G - 1)) == 0, "level %zu: %u groups", v, G);
        CHECK(cp.gp[b + G] - cp.gp[b] >= G, "level %zu: fewer columns than groups", v);
        for (uint32_t g = 0; g < G; g++) {
            CHECK(cp.gp[b + g] < cp.gp[b + g + 1], "level %zu: empty group %u", v, g);
            for (uint32_t c = cp.gp[b + g]; c < cp.gp[b + g + 1]; c++) {
                const uint32_t k = cp.cols[c];
                CHECK(k < n && level[k] < 0, "column %u twice", k);
                level[k] = (int)v;
                count++;
            }
        }
    }
    CHECK(count == n, "%zu of %u columns", count, n);
    for (uint32_t k = 0; k < n; k++)
        for (uint32_t p = t.up[k]; p < t.up[k + 1]; p++)
            CHECK(level[t.ui[p]] < level[k], "column %u reads column %u of its own level or later", k, t.ui[p]);
    CHECK(cp.ustream.size() == 4 * t.ui.size(), "entry stream size");
    for (size_t p = 0; p < t.ui.size(); p++) {
        const uint32_t i = t.ui[p];
        CHECK(cp.ustream[4 * p] == i && cp.ustream[4 * p + 1] == t.lp[i] && cp.ustream[4 * p + 2] == t.lp[i + 1],
              "entry stream %zu", p);
    }
    std::printf("columns: %zu levels\n", cp.lv_ptr.size() - 1);
}

int main(int argc, char** argv) {
    if (argc != 9) return 2;
    const auto cp = as<uint32_t>(slurp(argv[1])), ri = as<uint32_t>(slurp(argv[2])), q = as<uint32_t>(slurp(argv[4]));
    const auto v = as<double>(slurp(argv[3]));
    const uint32_t chunk = (uint32_t)std::atoi(argv[5]), rows = (uint32_t)std::atoi(argv[6]);
    const uint32_t ahead = (uint32_t)std::atoi(argv[7]), groups = (uint32_t)std::atoi(argv[8]);
    if (cp.size() < 2) return 2;
    const uint32_t n = (uint32_t)cp.size() - 1;
    Tape t;
    if (!factor_tape(n, cp.data(), ri.data(), v.data(), q, t)) return 3;
    LevelPlan lp;
    level_plan(t, lp);
    check_stream("forward", lp.fl_ptr, lp.fl_rows, lp.rl_ptr, lp.rl_ent, true, chunk, rows, ahead);
    check_stream("backward", lp.bl_ptr, lp.bl_rows, lp.ru_ptr, lp.ru_ent, false, chunk, rows, ahead);
    check_columns(t, groups);
    return fails ? 1 : 0;
}
