// Flattening of H-matrix / uniform-H descriptors into the slab layout and
// the N-form / T-form work lists (layout.hpp).  Runs once per matrix on the
// host; the result is uploaded as one device arena.
#include "plan.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>

#include <omp.h>

#include "common.hpp"

namespace hlrc {

namespace {

constexpr int64_t TFORM_TARGET_ELEMS = 8192;  // elements per T-form unit (64 KB FP64)

inline int64_t pad_rows(int64_t r) { return (r + 1) & ~int64_t(1); }  // 16-byte FP64 columns

struct Tiles {
    std::vector<int64_t> b;  // boundaries, ntiles + 1 entries
    int64_t n() const { return int64_t(b.size()) - 1; }
    int64_t first(int64_t lo) const { return int64_t(std::lower_bound(b.begin(), b.end(), lo) - b.begin()); }
    int64_t lo(int64_t i) const { return b[size_t(i)]; }
    int64_t size(int64_t i) const { return b[size_t(i + 1)] - b[size_t(i)]; }
};

// Output tiles: every block boundary is a tile boundary; gaps longer than
// TILE are split into near-equal pieces.
Tiles make_tiles(int64_t n, std::vector<int64_t> cuts) {
    cuts.push_back(0);
    cuts.push_back(n);
    std::sort(cuts.begin(), cuts.end());
    cuts.erase(std::unique(cuts.begin(), cuts.end()), cuts.end());
    Tiles t;
    t.b.push_back(0);
    for (size_t i = 0; i + 1 < cuts.size(); ++i) {
        const int64_t lo = cuts[i], gap = cuts[i + 1] - cuts[i];
        if (gap <= 0) continue;
        const int64_t pieces = (gap + TILE - 1) / TILE;
        const int64_t base = gap / pieces, rem = gap % pieces;
        int64_t pos = lo;
        for (int64_t p = 0; p < pieces; ++p) {
            pos += base + (p < rem ? 1 : 0);
            t.b.push_back(pos);
        }
    }
    return t;
}

struct CopyJob {
    int64_t dst;          // element offset in the store
    const double* src;    // column-major source
    int64_t lds, r0, rows, ncols, ld;
};

struct Store {
    std::vector<CopyJob> jobs;
    int64_t size = 0;
    int64_t alloc(const double* src, int64_t lds, int64_t r0, int64_t rows, int64_t ncols) {
        const int64_t ld = pad_rows(rows);
        const int64_t off = size;
        size += ld * ncols;
        jobs.push_back({off, src, lds, r0, rows, ncols, ld});
        return off;
    }
    void fill(std::vector<double>& st) const {
        st.assign(size_t(size), 0.0);
        #pragma omp parallel for schedule(dynamic, 64)
        for (int64_t i = 0; i < int64_t(jobs.size()); ++i) {
            const CopyJob& j = jobs[size_t(i)];
            for (int64_t c = 0; c < j.ncols; ++c)
                std::memcpy(st.data() + j.dst + c * j.ld, j.src + j.r0 + c * j.lds, size_t(j.rows) * sizeof(double));
        }
    }
};

inline int tclass(int nc) { return nc <= 8 ? 0 : (nc <= 16 ? 1 : 2); }

struct TBuilder {
    TPass& P;
    std::vector<std::pair<int64_t, TUnit>> tmp[3];  // (cost, unit) per class
    explicit TBuilder(TPass& p) : P(p) {}

    // one output of `ncols` columns at `out`, fed by `slabs`
    void add(uint32_t out, int64_t ncols, const std::vector<TSlab>& slabs) {
        for (const TSlab& s : slabs) P.alg_bytes += int64_t(sizeof(double)) * s.rows * (ncols + 1);
        P.alg_bytes += int64_t(sizeof(double)) * ncols * (P.mode == OUT_ADD_ALPHA ? 2 : 1);
        for (int64_t c0 = 0; c0 < ncols; c0 += TCOLS) {
            const int nc = int(std::min<int64_t>(TCOLS, ncols - c0));
            std::vector<std::pair<uint32_t, uint32_t>> runs;
            uint32_t sb = uint32_t(P.slabs.size());
            int64_t elems = 0;
            for (const TSlab& s : slabs) {
                P.slabs.push_back(s);
                elems += int64_t(s.rows) * nc;
                if (elems >= TFORM_TARGET_ELEMS) {
                    runs.push_back({sb, uint32_t(P.slabs.size())});
                    sb = uint32_t(P.slabs.size());
                    elems = 0;
                }
            }
            if (sb != uint32_t(P.slabs.size()) || runs.empty()) runs.push_back({sb, uint32_t(P.slabs.size())});
            if (runs.size() == 1) {
                TUnit u{runs[0].first, runs[0].second, uint32_t(out + c0), 0, uint8_t(nc), TU_DIRECT};
                u.c0 = uint16_t(c0);
                tmp[tclass(nc)].push_back({cost(u), u});
            } else {
                TGroup g{P.nslots, uint32_t(runs.size()), uint32_t(out + c0), uint32_t(nc)};
                P.groups.push_back(g);
                for (auto& r : runs) {
                    TUnit u{r.first, r.second, P.nslots++, uint16_t(c0), uint8_t(nc), 0};
                    tmp[tclass(nc)].push_back({cost(u), u});
                }
            }
        }
    }
    int64_t cost(const TUnit& u) const {
        int64_t e = 0;
        for (uint32_t s = u.sb; s < u.se; ++s) e += P.slabs[s].ld;
        return e * u.nc;
    }
    void finish() {
        P.units.clear();
        for (int c = 0; c < 3; ++c) {
            std::stable_sort(tmp[c].begin(), tmp[c].end(),
                             [](const auto& a, const auto& b) { return a.first > b.first; });
            P.cls_begin[c] = int(P.units.size());
            for (auto& e : tmp[c]) {
                P.units.push_back(e.second);
                P.bytes += e.first * int64_t(sizeof(double));
            }
        }
        P.cls_begin[3] = int(P.units.size());
    }
};

struct NBuilder {
    NPass& P;
    std::vector<std::pair<int64_t, NSeg>> tmp;
    explicit NBuilder(NPass& p) : P(p) {}
    uint32_t cb = 0;
    int64_t elems = 0, rows = 0, alg = 0;
    void begin(int64_t tile_rows) { cb = uint32_t(P.chunks.size()); elems = 0; rows = tile_rows; alg = 0; }
    void slab(int64_t off, int64_t ld, int64_t ncols, uint32_t vbase) {
        for (int64_t j0 = 0; j0 < ncols; j0 += NCHUNK) {
            const int nc = int(std::min<int64_t>(NCHUNK, ncols - j0));
            NChunk c{uint64_t(off + j0 * ld), uint32_t(vbase + uint32_t(j0)), uint16_t(nc), 0};
            P.chunks.push_back(c);
            elems += ld * nc;
        }
        alg += int64_t(sizeof(double)) * ncols * (rows + 1);
    }
    void end(uint32_t out, int64_t rows_, bool keep_empty) {
        const uint32_t ce = uint32_t(P.chunks.size());
        if (ce == cb && !keep_empty) return;
        NSeg s{cb, ce, out, uint16_t(rows_), uint16_t(pad_rows(rows_))};
        tmp.push_back({elems, s});
        P.alg_bytes += alg + int64_t(sizeof(double)) * rows_ * (P.mode == OUT_ADD_ALPHA ? 2 : 1);
    }
    void finish() {
        std::stable_sort(tmp.begin(), tmp.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
        P.segs.clear();
        for (auto& e : tmp) {
            P.segs.push_back(e.second);
            P.bytes += e.first * int64_t(sizeof(double));
        }
    }
};

// Tile T-form pass: objects (low-rank blocks / cluster bases) own an output
// of `ncols` coefficients and are cut into slabs by input tiles.  Objects on
// one tile write their chunks' results directly; objects on several tiles
// write per-tile partials that a finish pass sums in tile order.
struct TTBuilder {
    TTPass& P;
    std::vector<std::pair<int64_t, TTSeg>> tmp;
    std::vector<int64_t> pbase, ncol;
    std::vector<uint32_t> oout;
    uint32_t cb = 0, voff = 0;
    int64_t elems = 0, rows = 0;
    TTBuilder(TTPass& p, size_t nobj) : P(p), pbase(nobj, -2), ncol(nobj, 0), oout(nobj, 0) {}

    void object(size_t id, uint32_t out, int64_t ncols, int64_t ntiles) {
        ncol[id] = ncols;
        oout[id] = out;
        if (ntiles > 1) {
            pbase[id] = P.npart;
            P.groups.push_back({uint32_t(P.npart), uint32_t(ntiles), out, uint32_t(ncols)});
            P.npart += ntiles * ncols;
        } else {
            pbase[id] = -1;
        }
        P.alg_bytes += int64_t(sizeof(double)) * ncols * (P.mode == OUT_ADD_ALPHA ? 2 : 1);
    }
    void begin(int64_t v_off, int64_t tile_rows) {
        cb = uint32_t(P.chunks.size());
        voff = uint32_t(v_off);
        rows = tile_rows;
        elems = 0;
    }
    void slab(int64_t off, int64_t ld, size_t id, int64_t tile_idx) {
        const int64_t k = ncol[id];
        for (int64_t j0 = 0; j0 < k; j0 += TCOLS) {
            const int nc = int(std::min<int64_t>(TCOLS, k - j0));
            TTChunk c;
            c.a_off = uint64_t(off + j0 * ld);
            c.nc = uint16_t(nc);
            if (pbase[id] < 0) { c.out = uint32_t(oout[id] + j0); c.flags = TT_DIRECT; }
            else { c.out = uint32_t(pbase[id] + tile_idx * k + j0); c.flags = 0; }
            P.chunks.push_back(c);
            elems += ld * nc;
        }
        P.alg_bytes += int64_t(sizeof(double)) * rows * k;
    }
    void end() {
        const uint32_t ce = uint32_t(P.chunks.size());
        if (ce == cb) return;
        tmp.push_back({elems, TTSeg{cb, ce, voff, uint16_t(rows), uint16_t(pad_rows(rows))}});
        P.alg_bytes += int64_t(sizeof(double)) * rows;
    }
    void finish() {
        std::stable_sort(tmp.begin(), tmp.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
        P.segs.clear();
        for (auto& e : tmp) {
            P.segs.push_back(e.second);
            P.bytes += e.first * int64_t(sizeof(double));
        }
    }
};

inline double flops_gemv(double m, double n) { return 2.0 * m * n + 2.0 * m; }

}  // namespace

// --------------------------------------------------------------------- H
hlrc_status plan_h(const hlrc_h_desc& d, const hlrc_options& o, Plan& p) {
    if (d.nrows < 0 || d.ncols < 0 || d.nblocks < 0) return fail(HLRC_ERR_SHAPE, "negative matrix size");
    if (d.nblocks > 0 && !d.blocks) return fail(HLRC_ERR_ARG, "blocks == NULL");
    if (d.nrows >= (int64_t(1) << 31) || d.ncols >= (int64_t(1) << 31))
        return fail(HLRC_ERR_SHAPE, "matrix dimension exceeds 2^31-1");
    if (o.precision != HLRC_PREC_F64)
        return fail(HLRC_ERR_ARG, "precision %d not supported by this planner", o.precision);
    p = Plan();
    p.kind = 0;
    p.precision = o.precision;
    p.nrows = d.nrows;
    p.ncols = d.ncols;
    const int64_t nb = d.nblocks;
    double area = 0;
    std::vector<int64_t> rcuts, ccuts;
    for (int64_t i = 0; i < nb; ++i) {
        const hlrc_block& b = d.blocks[i];
        if (b.nrows < 0 || b.ncols < 0 || b.row0 < 0 || b.col0 < 0 || b.row0 + b.nrows > d.nrows ||
            b.col0 + b.ncols > d.ncols)
            return fail(HLRC_ERR_SHAPE, "block %lld: index set outside the matrix", (long long)i);
        if (b.kind == HLRC_LEAF_DENSE) {
            if (b.nrows * b.ncols > 0 && (!b.D || b.ldd < b.nrows))
                return fail(HLRC_ERR_ARG, "block %lld: dense data missing or ldd < nrows", (long long)i);
        } else if (b.kind == HLRC_LEAF_LOWRANK) {
            if (b.rank < 0) return fail(HLRC_ERR_SHAPE, "block %lld: negative rank", (long long)i);
            if (b.rank > 0 && ((b.nrows > 0 && (!b.U || b.ldu < b.nrows)) || (b.ncols > 0 && (!b.V || b.ldv < b.ncols))))
                return fail(HLRC_ERR_ARG, "block %lld: low-rank factors missing or bad leading dimension", (long long)i);
            if (b.rank > 65535) return fail(HLRC_ERR_SHAPE, "block %lld: rank above 65535", (long long)i);
        } else {
            return fail(HLRC_ERR_ARG, "block %lld: unknown leaf kind %d", (long long)i, b.kind);
        }
        area += double(b.nrows) * double(b.ncols);
        rcuts.push_back(b.row0);
        rcuts.push_back(b.row0 + b.nrows);
        ccuts.push_back(b.col0);
        ccuts.push_back(b.col0 + b.ncols);
    }
    if (area != double(d.nrows) * double(d.ncols))
        return fail(HLRC_ERR_SHAPE, "leaf blocks cover %.0f entries, matrix has %.0f (gap or overlap)", area,
                    double(d.nrows) * double(d.ncols));
    const Tiles tr = make_tiles(d.nrows, rcuts), tc = make_tiles(d.ncols, ccuts);
    p.n_row_tiles = tr.n();
    p.n_col_tiles = tc.n();

    // coefficient offsets and per-tile block lists (block order preserved)
    std::vector<int64_t> toff(size_t(nb), -1);
    int64_t nt = 0;
    std::vector<std::vector<int64_t>> rowlist(size_t(tr.n())), collist(size_t(tc.n()));
    for (int64_t i = 0; i < nb; ++i) {
        const hlrc_block& b = d.blocks[i];
        if (b.nrows == 0 || b.ncols == 0) continue;
        const bool lr = b.kind == HLRC_LEAF_LOWRANK;
        if (lr && b.rank == 0) continue;
        if (lr) { toff[i] = nt; nt += b.rank; }
        for (int64_t t = tr.first(b.row0); t < tr.first(b.row0 + b.nrows); ++t) rowlist[size_t(t)].push_back(i);
        for (int64_t t = tc.first(b.col0); t < tc.first(b.col0 + b.ncols); ++t) collist[size_t(t)].push_back(i);
    }
    if (nt >= (int64_t(1) << 31)) return fail(HLRC_ERR_SHAPE, "sum of ranks exceeds 2^31-1");
    p.n_t = nt;

    // storage: row region (per row tile: D and U slabs), then V region
    Store st;
    std::vector<std::vector<int64_t>> slabA(static_cast<size_t>(nb)), slabV(static_cast<size_t>(nb));  // A = D or U, by row tile
    for (int64_t t = 0; t < tr.n(); ++t) {
        for (int64_t i : rowlist[size_t(t)]) {
            const hlrc_block& b = d.blocks[i];
            const int64_t r0 = tr.lo(t) - b.row0, rows = tr.size(t);
            if (b.kind == HLRC_LEAF_DENSE) slabA[size_t(i)].push_back(st.alloc(b.D, b.ldd, r0, rows, b.ncols));
            else slabA[size_t(i)].push_back(st.alloc(b.U, b.ldu, r0, rows, b.rank));
        }
    }
    // V slabs ordered by column tile, so that stage A of op N streams one
    // contiguous region per tile
    for (int64_t t = 0; t < tc.n(); ++t)
        for (int64_t i : collist[size_t(t)]) {
            const hlrc_block& b = d.blocks[i];
            if (b.kind != HLRC_LEAF_LOWRANK) continue;
            slabV[size_t(i)].push_back(st.alloc(b.V, b.ldv, tc.lo(t) - b.col0, tc.size(t), b.rank));
        }
    st.fill(p.store);

    // op N: tile T-form V^T x -> t (per column tile), then N-form per row tile: U t + D x -> y
    p.tpasses.resize(1);
    p.npasses.resize(2);
    p.ttpasses.resize(2);
    {
        TTPass& a = p.ttpasses[0];
        a.in = V_X; a.out = V_T; a.mode = OUT_SET;
        TTBuilder tb(a, size_t(nb));
        for (int64_t i = 0; i < nb; ++i)
            if (toff[size_t(i)] >= 0)
                tb.object(size_t(i), uint32_t(toff[size_t(i)]), d.blocks[i].rank,
                          tc.first(d.blocks[i].col0 + d.blocks[i].ncols) - tc.first(d.blocks[i].col0));
        for (int64_t t = 0; t < tc.n(); ++t) {
            tb.begin(tc.lo(t), tc.size(t));
            const int64_t ld = pad_rows(tc.size(t));
            for (int64_t i : collist[size_t(t)]) {
                if (toff[size_t(i)] < 0) continue;
                const int64_t ti = t - tc.first(d.blocks[i].col0);
                tb.slab(slabV[size_t(i)][size_t(ti)], ld, size_t(i), ti);
            }
            tb.end();
        }
        tb.finish();
    }
    {
        NPass& nN = p.npasses[0];
        nN.vx = V_X; nN.vt = V_T; nN.out = V_Y; nN.mode = OUT_ADD_ALPHA;
        NBuilder nbld(nN);
        std::vector<size_t> pos(size_t(nb), 0);
        for (int64_t t = 0; t < tr.n(); ++t) {
            nbld.begin(tr.size(t));
            const int64_t ld = pad_rows(tr.size(t));
            for (int64_t i : rowlist[size_t(t)]) {
                const hlrc_block& b = d.blocks[i];
                const int64_t off = slabA[size_t(i)][pos[size_t(i)]++];
                if (b.kind == HLRC_LEAF_DENSE) nbld.slab(off, ld, b.ncols, uint32_t(b.col0));
                else nbld.slab(off, ld, b.rank, VEC_T | uint32_t(toff[size_t(i)]));
            }
            nbld.end(uint32_t(tr.lo(t)), tr.size(t), false);
        }
        nbld.finish();
    }
    // op T: tile T-form U^T x -> t (per row tile); N-form per column tile V t -> y; T-form D^T x -> y
    {
        TTPass& a = p.ttpasses[1];
        a.in = V_X; a.out = V_T; a.mode = OUT_SET;
        TTBuilder tb(a, size_t(nb));
        for (int64_t i = 0; i < nb; ++i)
            if (toff[size_t(i)] >= 0)
                tb.object(size_t(i), uint32_t(toff[size_t(i)]), d.blocks[i].rank,
                          tr.first(d.blocks[i].row0 + d.blocks[i].nrows) - tr.first(d.blocks[i].row0));
        for (int64_t t = 0; t < tr.n(); ++t) {
            tb.begin(tr.lo(t), tr.size(t));
            const int64_t ld = pad_rows(tr.size(t));
            for (int64_t i : rowlist[size_t(t)]) {
                if (toff[size_t(i)] < 0) continue;
                const int64_t ti = t - tr.first(d.blocks[i].row0);
                tb.slab(slabA[size_t(i)][size_t(ti)], ld, size_t(i), ti);
            }
            tb.end();
        }
        tb.finish();
    }
    {
        NPass& nT = p.npasses[1];
        nT.vx = V_X; nT.vt = V_T; nT.out = V_Y; nT.mode = OUT_ADD_ALPHA;
        NBuilder nbld(nT);
        for (int64_t t = 0; t < tc.n(); ++t) {
            nbld.begin(tc.size(t));
            const int64_t ld = pad_rows(tc.size(t));
            for (int64_t i : collist[size_t(t)]) {
                const hlrc_block& b = d.blocks[i];
                if (b.kind != HLRC_LEAF_LOWRANK) continue;
                const int64_t off = slabV[size_t(i)][size_t(t - tc.first(b.col0))];
                nbld.slab(off, ld, b.rank, VEC_T | uint32_t(toff[size_t(i)]));
            }
            nbld.end(uint32_t(tc.lo(t)), tc.size(t), false);
        }
        nbld.finish();
    }
    {
        TPass& dT = p.tpasses[0];
        dT.in = V_X; dT.out = V_Y; dT.mode = OUT_ADD_ALPHA;
        TBuilder tb(dT);
        for (int64_t t = 0; t < tc.n(); ++t) {
            std::vector<TSlab> sl;
            for (int64_t i : collist[size_t(t)]) {
                const hlrc_block& b = d.blocks[i];
                if (b.kind != HLRC_LEAF_DENSE) continue;
                const int64_t r0 = tr.first(b.row0);
                for (size_t s = 0; s < slabA[size_t(i)].size(); ++s) {
                    const int64_t rt = r0 + int64_t(s);
                    const int64_t ld = pad_rows(tr.size(rt));
                    sl.push_back({uint64_t(slabA[size_t(i)][s] + (tc.lo(t) - b.col0) * ld), uint32_t(tr.lo(rt)),
                                  uint16_t(tr.size(rt)), uint16_t(ld)});
                }
            }
            if (!sl.empty()) tb.add(uint32_t(tc.lo(t)), tc.size(t), sl);
        }
        tb.finish();
    }
    p.stages[HLRC_OP_N] = {{2, 0}, {1, 0}};
    p.stages[HLRC_OP_T] = {{2, 1}, {1, 1}, {0, 0}};
    p.stages[HLRC_OP_C] = p.stages[HLRC_OP_T];
    for (const TTPass& tp : p.ttpasses)
        if (tp.npart >= (int64_t(1) << 32)) return fail(HLRC_ERR_SHAPE, "partial array exceeds 2^32 entries");

    // accounting (arith/mulvec.hh:795-874)
    double flops = 0, mbytes = 0;
    for (int64_t i = 0; i < nb; ++i) {
        const hlrc_block& b = d.blocks[i];
        if (b.kind == HLRC_LEAF_DENSE) {
            ++p.n_dense;
            flops += flops_gemv(double(b.nrows), double(b.ncols));
            mbytes += 8.0 * double(b.nrows) * double(b.ncols);
        } else {
            ++p.n_lowrank;
            flops += flops_gemv(double(b.ncols), b.rank) + flops_gemv(double(b.nrows), b.rank);
            mbytes += 8.0 * double(b.rank) * double(b.nrows + b.ncols);
            p.max_rank = std::max(p.max_rank, b.rank);
        }
    }
    p.matrix_bytes = int64_t(mbytes);
    p.algorithmic_bytes = int64_t(mbytes) + 2 * 8 * (d.nrows + d.ncols);
    p.flops = int64_t(flops);
    return HLRC_OK;
}

// ------------------------------------------------------------- uniform-H
hlrc_status plan_uniform(const hlrc_uniform_desc& d, const hlrc_options& o, Plan& p) {
    if (d.nrows < 0 || d.ncols < 0 || d.nblocks < 0 || d.nrow_bases < 0 || d.ncol_bases < 0)
        return fail(HLRC_ERR_SHAPE, "negative size");
    if ((d.nblocks > 0 && !d.blocks) || (d.nrow_bases > 0 && !d.row_bases) || (d.ncol_bases > 0 && !d.col_bases))
        return fail(HLRC_ERR_ARG, "NULL array in uniform descriptor");
    if (d.nrows >= (int64_t(1) << 31) || d.ncols >= (int64_t(1) << 31))
        return fail(HLRC_ERR_SHAPE, "matrix dimension exceeds 2^31-1");
    if (o.precision != HLRC_PREC_F64)
        return fail(HLRC_ERR_ARG, "precision %d not supported for uniform-H", o.precision);
    p = Plan();
    p.kind = 1;
    p.precision = o.precision;
    p.nrows = d.nrows;
    p.ncols = d.ncols;
    const int64_t nb = d.nblocks, nrb = d.nrow_bases, ncb = d.ncol_bases;
    auto check_basis = [&](const hlrc_basis& b, int64_t n) {
        return b.ofs >= 0 && b.size >= 0 && b.ofs + b.size <= n && b.rank >= 0 && b.rank <= 65535 &&
               (b.rank == 0 || b.size == 0 || (b.V && b.ldv >= b.size));
    };
    for (int64_t i = 0; i < nrb; ++i)
        if (!check_basis(d.row_bases[i], d.nrows)) return fail(HLRC_ERR_SHAPE, "row basis %lld invalid", (long long)i);
    for (int64_t i = 0; i < ncb; ++i)
        if (!check_basis(d.col_bases[i], d.ncols)) return fail(HLRC_ERR_SHAPE, "column basis %lld invalid", (long long)i);
    double area = 0;
    std::vector<int64_t> rcuts, ccuts;
    for (int64_t i = 0; i < nb; ++i) {
        const hlrc_uniform_block& b = d.blocks[i];
        if (b.nrows < 0 || b.ncols < 0 || b.row0 < 0 || b.col0 < 0 || b.row0 + b.nrows > d.nrows ||
            b.col0 + b.ncols > d.ncols)
            return fail(HLRC_ERR_SHAPE, "block %lld: index set outside the matrix", (long long)i);
        if (b.kind == HLRC_LEAF_DENSE) {
            if (b.nrows * b.ncols > 0 && (!b.D || b.ldd < b.nrows))
                return fail(HLRC_ERR_ARG, "block %lld: dense data missing", (long long)i);
        } else if (b.kind == HLRC_LEAF_LOWRANK) {
            if (b.row_basis < 0 || b.row_basis >= nrb || b.col_basis < 0 || b.col_basis >= ncb)
                return fail(HLRC_ERR_ARG, "block %lld: basis index out of range", (long long)i);
            const hlrc_basis& rb = d.row_bases[b.row_basis];
            const hlrc_basis& cb = d.col_bases[b.col_basis];
            if (rb.ofs != b.row0 || rb.size != b.nrows || cb.ofs != b.col0 || cb.size != b.ncols)
                return fail(HLRC_ERR_SHAPE, "block %lld: basis index sets differ from the block's", (long long)i);
            if (rb.rank > 0 && cb.rank > 0 && (!b.S || b.lds < rb.rank))
                return fail(HLRC_ERR_ARG, "block %lld: coupling missing or lds < row rank", (long long)i);
        } else {
            return fail(HLRC_ERR_ARG, "block %lld: unknown kind", (long long)i);
        }
        area += double(b.nrows) * double(b.ncols);
        rcuts.push_back(b.row0); rcuts.push_back(b.row0 + b.nrows);
        ccuts.push_back(b.col0); ccuts.push_back(b.col0 + b.ncols);
    }
    if (area != double(d.nrows) * double(d.ncols))
        return fail(HLRC_ERR_SHAPE, "leaf blocks cover %.0f entries, matrix has %.0f", area,
                    double(d.nrows) * double(d.ncols));
    for (int64_t i = 0; i < nrb; ++i) { rcuts.push_back(d.row_bases[i].ofs); rcuts.push_back(d.row_bases[i].ofs + d.row_bases[i].size); }
    for (int64_t i = 0; i < ncb; ++i) { ccuts.push_back(d.col_bases[i].ofs); ccuts.push_back(d.col_bases[i].ofs + d.col_bases[i].size); }
    const Tiles tr = make_tiles(d.nrows, rcuts), tc = make_tiles(d.ncols, ccuts);
    p.n_row_tiles = tr.n();
    p.n_col_tiles = tc.n();

    std::vector<int64_t> rboff(size_t(nrb), -1), cboff(size_t(ncb), -1);
    int64_t nkr = 0, nkc = 0;
    for (int64_t i = 0; i < nrb; ++i)
        if (d.row_bases[i].rank > 0 && d.row_bases[i].size > 0) { rboff[size_t(i)] = nkr; nkr += d.row_bases[i].rank; }
    for (int64_t i = 0; i < ncb; ++i)
        if (d.col_bases[i].rank > 0 && d.col_bases[i].size > 0) { cboff[size_t(i)] = nkc; nkc += d.col_bases[i].rank; }
    if (std::max(nkr, nkc) >= (int64_t(1) << 31)) return fail(HLRC_ERR_SHAPE, "sum of basis ranks exceeds 2^31-1");
    p.n_t = std::max(nkr, nkc);
    p.n_t2 = std::max(nkr, nkc);

    // tile -> bases / dense blocks covering it
    std::vector<std::vector<int64_t>> rbl(size_t(tr.n())), cbl(size_t(tc.n())), rdl(size_t(tr.n())), cdl(size_t(tc.n()));
    for (int64_t i = 0; i < nrb; ++i)
        if (rboff[size_t(i)] >= 0)
            for (int64_t t = tr.first(d.row_bases[i].ofs); t < tr.first(d.row_bases[i].ofs + d.row_bases[i].size); ++t)
                rbl[size_t(t)].push_back(i);
    for (int64_t i = 0; i < ncb; ++i)
        if (cboff[size_t(i)] >= 0)
            for (int64_t t = tc.first(d.col_bases[i].ofs); t < tc.first(d.col_bases[i].ofs + d.col_bases[i].size); ++t)
                cbl[size_t(t)].push_back(i);
    std::vector<std::vector<int64_t>> lr_by_row(static_cast<size_t>(nrb)), lr_by_col(static_cast<size_t>(ncb));
    for (int64_t i = 0; i < nb; ++i) {
        const hlrc_uniform_block& b = d.blocks[i];
        if (b.nrows == 0 || b.ncols == 0) continue;
        if (b.kind == HLRC_LEAF_DENSE) {
            for (int64_t t = tr.first(b.row0); t < tr.first(b.row0 + b.nrows); ++t) rdl[size_t(t)].push_back(i);
            for (int64_t t = tc.first(b.col0); t < tc.first(b.col0 + b.ncols); ++t) cdl[size_t(t)].push_back(i);
        } else {
            if (rboff[size_t(b.row_basis)] < 0 || cboff[size_t(b.col_basis)] < 0) continue;
            lr_by_row[size_t(b.row_basis)].push_back(i);
            lr_by_col[size_t(b.col_basis)].push_back(i);
        }
    }

    Store st;
    std::vector<std::vector<int64_t>> sRB(static_cast<size_t>(nrb)), sCB(static_cast<size_t>(ncb)), sD(static_cast<size_t>(nb)), sS(static_cast<size_t>(nb));
    for (int64_t t = 0; t < tr.n(); ++t) {
        for (int64_t i : rbl[size_t(t)]) {
            const hlrc_basis& b = d.row_bases[i];
            sRB[size_t(i)].push_back(st.alloc(b.V, b.ldv, tr.lo(t) - b.ofs, tr.size(t), b.rank));
        }
        for (int64_t i : rdl[size_t(t)]) {
            const hlrc_uniform_block& b = d.blocks[i];
            sD[size_t(i)].push_back(st.alloc(b.D, b.ldd, tr.lo(t) - b.row0, tr.size(t), b.ncols));
        }
    }
    for (int64_t t = 0; t < tc.n(); ++t)   // column bases by column tile
        for (int64_t i : cbl[size_t(t)]) {
            const hlrc_basis& b = d.col_bases[i];
            sCB[size_t(i)].push_back(st.alloc(b.V, b.ldv, tc.lo(t) - b.ofs, tc.size(t), b.rank));
        }
    for (int64_t i = 0; i < nb; ++i) {
        const hlrc_uniform_block& b = d.blocks[i];
        if (b.kind != HLRC_LEAF_LOWRANK || b.nrows == 0 || b.ncols == 0) continue;
        if (rboff[size_t(b.row_basis)] < 0 || cboff[size_t(b.col_basis)] < 0) continue;
        const int64_t kr = d.row_bases[b.row_basis].rank, kc = d.col_bases[b.col_basis].rank;
        for (int64_t r0 = 0; r0 < kr; r0 += TILE)
            sS[size_t(i)].push_back(st.alloc(b.S, b.lds, r0, std::min<int64_t>(TILE, kr - r0), kc));
    }
    st.fill(p.store);

    p.tpasses.resize(4);
    p.npasses.resize(3);
    p.ttpasses.resize(2);
    // ---- op N
    {   // forward: ux_s = V_s^T x, per column tile over all bases containing it
        TTPass& f = p.ttpasses[0];
        f.in = V_X; f.out = V_T; f.mode = OUT_SET;
        TTBuilder tb(f, size_t(ncb));
        for (int64_t i = 0; i < ncb; ++i)
            if (cboff[size_t(i)] >= 0)
                tb.object(size_t(i), uint32_t(cboff[size_t(i)]), d.col_bases[i].rank,
                          tc.first(d.col_bases[i].ofs + d.col_bases[i].size) - tc.first(d.col_bases[i].ofs));
        for (int64_t t = 0; t < tc.n(); ++t) {
            tb.begin(tc.lo(t), tc.size(t));
            const int64_t ld = pad_rows(tc.size(t));
            for (int64_t i : cbl[size_t(t)]) {
                const int64_t ti = t - tc.first(d.col_bases[i].ofs);
                tb.slab(sCB[size_t(i)][size_t(ti)], ld, size_t(i), ti);
            }
            tb.end();
        }
        tb.finish();
    }
    {   // coupling: uy_t = sum_s S_ts ux_s
        NPass& c = p.npasses[0];
        c.vx = V_X; c.vt = V_T; c.out = V_T2; c.mode = OUT_SET;
        NBuilder nbld(c);
        for (int64_t t = 0; t < nrb; ++t) {
            if (rboff[size_t(t)] < 0) continue;
            const int64_t kr = d.row_bases[t].rank;
            for (int64_t r0 = 0, piece = 0; r0 < kr; r0 += TILE, ++piece) {
                nbld.begin(std::min<int64_t>(TILE, kr - r0));
                const int64_t rows = std::min<int64_t>(TILE, kr - r0);
                for (int64_t i : lr_by_row[size_t(t)]) {
                    const hlrc_uniform_block& b = d.blocks[i];
                    nbld.slab(sS[size_t(i)][size_t(piece)], pad_rows(rows), d.col_bases[b.col_basis].rank,
                              VEC_T | uint32_t(cboff[size_t(b.col_basis)]));
                }
                nbld.end(uint32_t(rboff[size_t(t)] + r0), rows, true);
            }
        }
        nbld.finish();
    }
    {   // backward + near field: y_tau += alpha (sum_t V_t[tau] uy_t + sum D x)
        NPass& bw = p.npasses[1];
        bw.vx = V_X; bw.vt = V_T2; bw.out = V_Y; bw.mode = OUT_ADD_ALPHA;
        NBuilder nbld(bw);
        std::vector<size_t> posRB(size_t(nrb), 0), posD(size_t(nb), 0);
        for (int64_t t = 0; t < tr.n(); ++t) {
            nbld.begin(tr.size(t));
            const int64_t ld = pad_rows(tr.size(t));
            for (int64_t i : rbl[size_t(t)])
                nbld.slab(sRB[size_t(i)][posRB[size_t(i)]++], ld, d.row_bases[i].rank, VEC_T | uint32_t(rboff[size_t(i)]));
            for (int64_t i : rdl[size_t(t)])
                nbld.slab(sD[size_t(i)][posD[size_t(i)]++], ld, d.blocks[i].ncols, uint32_t(d.blocks[i].col0));
            nbld.end(uint32_t(tr.lo(t)), tr.size(t), false);
        }
        nbld.finish();
    }
    // ---- op C (adjoint)
    {   // forward with row bases: ux'_t = V_t^T x, per row tile
        TTPass& f = p.ttpasses[1];
        f.in = V_X; f.out = V_T; f.mode = OUT_SET;
        TTBuilder tb(f, size_t(nrb));
        for (int64_t i = 0; i < nrb; ++i)
            if (rboff[size_t(i)] >= 0)
                tb.object(size_t(i), uint32_t(rboff[size_t(i)]), d.row_bases[i].rank,
                          tr.first(d.row_bases[i].ofs + d.row_bases[i].size) - tr.first(d.row_bases[i].ofs));
        for (int64_t t = 0; t < tr.n(); ++t) {
            tb.begin(tr.lo(t), tr.size(t));
            const int64_t ld = pad_rows(tr.size(t));
            for (int64_t i : rbl[size_t(t)]) {
                const int64_t ti = t - tr.first(d.row_bases[i].ofs);
                tb.slab(sRB[size_t(i)][size_t(ti)], ld, size_t(i), ti);
            }
            tb.end();
        }
        tb.finish();
    }
    {   // coupling^T: uy'_s = sum_t S_ts^T ux'_t
        TPass& c = p.tpasses[2];
        c.in = V_T; c.out = V_T2; c.mode = OUT_SET;
        TBuilder tb(c);
        for (int64_t s = 0; s < ncb; ++s) {
            if (cboff[size_t(s)] < 0) continue;
            std::vector<TSlab> sl;
            for (int64_t i : lr_by_col[size_t(s)]) {
                const hlrc_uniform_block& b = d.blocks[i];
                const int64_t kr = d.row_bases[b.row_basis].rank;
                for (int64_t r0 = 0, piece = 0; r0 < kr; r0 += TILE, ++piece) {
                    const int64_t rows = std::min<int64_t>(TILE, kr - r0);
                    sl.push_back({uint64_t(sS[size_t(i)][size_t(piece)]), uint32_t(rboff[size_t(b.row_basis)] + r0),
                                  uint16_t(rows), uint16_t(pad_rows(rows))});
                }
            }
            tb.add(uint32_t(cboff[size_t(s)]), d.col_bases[s].rank, sl);
        }
        tb.finish();
    }
    {   // backward with column bases: y_sigma += alpha sum_s V_s[sigma] uy'_s
        NPass& bw = p.npasses[2];
        bw.vx = V_X; bw.vt = V_T2; bw.out = V_Y; bw.mode = OUT_ADD_ALPHA;
        NBuilder nbld(bw);
        for (int64_t t = 0; t < tc.n(); ++t) {
            nbld.begin(tc.size(t));
            const int64_t ld = pad_rows(tc.size(t));
            for (int64_t i : cbl[size_t(t)])
                nbld.slab(sCB[size_t(i)][size_t(t - tc.first(d.col_bases[i].ofs))], ld, d.col_bases[i].rank,
                          VEC_T | uint32_t(cboff[size_t(i)]));
            nbld.end(uint32_t(tc.lo(t)), tc.size(t), false);
        }
        nbld.finish();
    }
    {   // near field transposed: y_sigma += alpha sum D^T x
        TPass& dT = p.tpasses[3];
        dT.in = V_X; dT.out = V_Y; dT.mode = OUT_ADD_ALPHA;
        TBuilder tb(dT);
        for (int64_t t = 0; t < tc.n(); ++t) {
            std::vector<TSlab> sl;
            for (int64_t i : cdl[size_t(t)]) {
                const hlrc_uniform_block& b = d.blocks[i];
                const int64_t r0 = tr.first(b.row0);
                for (size_t s = 0; s < sD[size_t(i)].size(); ++s) {
                    const int64_t rt = r0 + int64_t(s);
                    const int64_t ld = pad_rows(tr.size(rt));
                    sl.push_back({uint64_t(sD[size_t(i)][s] + (tc.lo(t) - b.col0) * ld), uint32_t(tr.lo(rt)),
                                  uint16_t(tr.size(rt)), uint16_t(ld)});
                }
            }
            if (!sl.empty()) tb.add(uint32_t(tc.lo(t)), tc.size(t), sl);
        }
        tb.finish();
    }
    p.stages[HLRC_OP_N] = {{2, 0}, {1, 0}, {1, 1}};
    p.stages[HLRC_OP_T].clear();  // uniform_lrmatrix::uni_apply_add asserts on apply_transposed
    p.stages[HLRC_OP_C] = {{2, 1}, {0, 2}, {1, 2}, {0, 3}};
    for (const TTPass& tp : p.ttpasses)
        if (tp.npart >= (int64_t(1) << 32)) return fail(HLRC_ERR_SHAPE, "partial array exceeds 2^32 entries");

    // accounting (arith/uniform.hh:285-325)
    double flops = 0, mbytes = 0, cbbytes = 0, rbbytes = 0;
    for (int64_t i = 0; i < ncb; ++i) {
        const auto& b = d.col_bases[i];
        if (b.rank > 0) { flops += flops_gemv(b.rank, double(b.size)); cbbytes += 8.0 * b.rank * double(b.size); }
    }
    for (int64_t i = 0; i < nrb; ++i) {
        const auto& b = d.row_bases[i];
        if (b.rank > 0) { flops += flops_gemv(double(b.size), b.rank); rbbytes += 8.0 * b.rank * double(b.size); }
        p.max_rank = std::max(p.max_rank, b.rank);
    }
    for (int64_t i = 0; i < nb; ++i) {
        const auto& b = d.blocks[i];
        if (b.kind == HLRC_LEAF_DENSE) {
            ++p.n_dense;
            flops += flops_gemv(double(b.nrows), double(b.ncols));
            mbytes += 8.0 * double(b.nrows) * double(b.ncols);
        } else {
            ++p.n_lowrank;
            const double kr = d.row_bases[b.row_basis].rank, kc = d.col_bases[b.col_basis].rank;
            flops += flops_gemv(kr, kc);
            mbytes += 8.0 * kr * kc;
        }
    }
    p.matrix_bytes = int64_t(mbytes + cbbytes + rbbytes);
    p.algorithmic_bytes = int64_t(cbbytes + 8.0 * d.ncols + mbytes + rbbytes + 8.0 * d.nrows);
    p.flops = int64_t(flops);
    return HLRC_OK;
}

}  // namespace hlrc
