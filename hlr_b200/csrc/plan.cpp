// Flattening of H-matrix / uniform-H descriptors into the slab layout and
// the N-form / tile-T-form work lists (layout.hpp).  Runs once per matrix on
// the host; the result is uploaded as one device arena.
#include "plan.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <numeric>
#include <unordered_map>

#include <omp.h>

#include "common.hpp"

namespace hlrc {

namespace {

constexpr int64_t TFORM_TARGET_ELEMS = 8192;  // elements per T-form unit (64 KB FP64)

inline int64_t pad_rows(int64_t r) { return (r + 1) & ~int64_t(1); }  // lanes own row pairs
inline int64_t align16(int64_t b) { return (b + 15) & ~int64_t(15); }

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

// ---- number formats (round to nearest even), written from the IEEE 754
// binary16 and bfloat16 definitions
uint16_t to_bf16(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    if ((u & 0x7f800000u) == 0x7f800000u) return uint16_t((u >> 16) | ((u & 0xffffu) ? 0x40u : 0u));  // inf / nan
    const uint32_t lsb = (u >> 16) & 1u;
    u += 0x7fffu + lsb;
    return uint16_t(u >> 16);
}

uint16_t to_f16(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    const uint32_t sign = (u >> 16) & 0x8000u;
    const int32_t exp = int32_t((u >> 23) & 0xff);
    uint32_t man = u & 0x7fffffu;
    if (exp == 0xff) return uint16_t(sign | 0x7c00u | (man ? 0x200u : 0u));
    int32_t e = exp - 127 + 15;
    if (e >= 0x1f) return uint16_t(sign | 0x7c00u);  // overflow -> inf
    if (e <= 0) {                                   // subnormal or zero
        if (e < -10) return uint16_t(sign);
        man |= 0x800000u;
        const int shift = 14 - e;                   // 24-bit mantissa -> 10 - (1 - e) bits
        const uint32_t half = 1u << (shift - 1);
        uint32_t r = man >> shift;
        const uint32_t rem = man & ((1u << shift) - 1u);
        if (rem > half || (rem == half && (r & 1u))) ++r;
        return uint16_t(sign | r);
    }
    uint32_t r = man >> 13;
    const uint32_t rem = man & 0x1fffu;
    if (rem > 0x1000u || (rem == 0x1000u && (r & 1u))) {
        ++r;
        if (r == 0x400u) { r = 0; ++e; if (e >= 0x1f) return uint16_t(sign | 0x7c00u); }
    }
    return uint16_t(sign | (uint32_t(e) << 10) | r);
}

// ---- store: slabs cut into chunks of one format.  A chunk holds at most
// 4 KB at full tile height (FP64: 8 columns, FP32: 16, 16-bit: 32) and its
// columns are padded so that every lane's 16-byte load is aligned: rows are
// padded to 2 (FP64), 4 (FP32) or 8 (16-bit).
inline int chunk_cols(int f) { return f == FMT_F64 ? 8 : (f == FMT_F32 ? 16 : 32); }
// 24-bit columns pad to 16 rows: the 8-byte low-part loads of a lane then
// start 16-byte aligned runs like the 16-byte high-part loads
inline int64_t pad_fmt(int64_t rows, int f) {
    const int64_t m = f == FMT_F64 ? 2 : (f == FMT_F32 ? 4 : (f == FMT_I24 ? 16 : 8));
    return (rows + m - 1) / m * m;
}

struct SChunk {
    int64_t byte_off;
    int32_t col0;
    int16_t nc;
    uint8_t fmt;
    float scale;
};

struct SSlab {
    const double* src;
    int64_t lds, r0, rows, ld;   // ld: FP64 padding (FP64 stores); chunks use pad_fmt(rows, fmt)
    int32_t c0, nch;             // chunks [c0, c0 + nch)
};

// Layout order of the chunks of one tile region: dense (D) or factor (U, V,
// bases) slabs, by format.  With it, every pass segment of one format is a
// contiguous run of columns in every store this planner produces: FP64 D,U;
// FP32 D,U; mixed D(FP32),U(FP32),U(FP16); FP16 / BF16 U,D.
inline int layout_rank(int group, int fmt) {
    static const int rank[NFMT][2] = {{0, 1}, {2, 3}, {5, 4}, {7, 6}, {9, 8}, {10, 11}};   // [fmt][group]: D = 0, factor = 1
    return rank[fmt][group];
}

struct Store {
    std::vector<SSlab> slabs;
    std::vector<SChunk> chunks;
    std::vector<uint8_t> group;        // per chunk: 0 = dense slab, 1 = factor slab
    std::vector<int32_t> crows;        // per chunk: rows of its slab
    // per chunk: scale group (-1: the chunk's own scale).  Scaled chunks of
    // one group share the scale of the group's largest entry.
    std::vector<int32_t> sgrp;
    // per chunk: row group (-1: none) and exponent c.  The chunks of a row
    // group get scale F 2^-c, where F is the largest of the chunks' own
    // scales times 2^c: one output tile's chunks then need no factors when
    // the vector entries of a chunk with exponent c are kept times 2^-c.
    std::vector<int32_t> rgrp;
    std::vector<int32_t> cexp;
    // 16-bit chunks of a region start each layout group on a 128-byte
    // boundary (full-height columns are then 128-byte rows for 2-D TMA)
    bool align128 = false;
    size_t region_begin = 0;           // first chunk without a byte offset
    int64_t bytes = 0;
    int64_t unpadded[NFMT] = {};

    // rows [r0, r0+rows) x ncols of a column-major matrix; colfmt (per
    // column, may be null -> deffmt); chunks do not straddle `cuts`.  Byte
    // offsets are assigned by close_region().
    int alloc(const double* src, int64_t lds, int64_t r0, int64_t rows, int64_t ncols, const uint8_t* colfmt,
              uint8_t deffmt, const std::vector<int64_t>* cuts = nullptr, int grp = 1, int32_t scale_group = -1,
              int32_t row_group = -1, int32_t c_exp = 0) {
        SSlab s{src, lds, r0, rows, pad_rows(rows), int32_t(chunks.size()), 0};
        int64_t j = 0;
        size_t ci = 0;
        while (j < ncols) {
            const uint8_t f = colfmt ? colfmt[j] : deffmt;
            int64_t e = std::min<int64_t>(j + chunk_cols(f), ncols);
            if (cuts) {
                while (ci < cuts->size() && (*cuts)[ci] <= j) ++ci;
                if (ci < cuts->size()) e = std::min<int64_t>(e, (*cuts)[ci]);
            }
            for (int64_t c = j + 1; c < e; ++c)
                if ((colfmt ? colfmt[c] : deffmt) != f) { e = c; break; }
            SChunk ch{-1, int32_t(j), int16_t(e - j), f, 1.0f};
            unpadded[f] += rows * (e - j) * fmt_bytes(f) + (f >= FMT_F16 ? 4 : 0);
            chunks.push_back(ch);
            group.push_back(uint8_t(grp));
            crows.push_back(int32_t(rows));
            sgrp.push_back(scale_group);
            rgrp.push_back(row_group);
            cexp.push_back(c_exp);
            ++s.nch;
            j = e;
        }
        slabs.push_back(s);
        return int(slabs.size()) - 1;
    }

    // Places the chunks allocated since the last call: by layout_rank, then
    // in allocation order, each on a 16-byte boundary.  With align128 the
    // region's first 16-bit chunk starts on a 128-byte boundary; the chunks
    // after it follow without a gap, since a pass segment may span the
    // factor and dense groups and must stay one contiguous column run.
    void close_region() {
        bool first16 = true;
        for (int r = 0; r < 2 * NFMT; ++r) {
            for (size_t c = region_begin; c < chunks.size(); ++c) {
                SChunk& ch = chunks[c];
                if (layout_rank(group[c], ch.fmt) != r) continue;
                ch.byte_off = align16(bytes);
                if (first16 && align128 && (ch.fmt == FMT_F16 || ch.fmt == FMT_BF16)) {
                    ch.byte_off = (ch.byte_off + 127) / 128 * 128;
                    first16 = false;
                }
                bytes = ch.byte_off + pad_fmt(crows[c], ch.fmt) * ch.nc * fmt_bytes(ch.fmt);
            }
        }
        region_begin = chunks.size();
    }

    // largest |entry| of each chunk's slab rows and columns
    double chunk_amax(const SSlab& s, const SChunk& ch) const {
        double amax = 0;
        const double* src = s.src + s.r0 + int64_t(ch.col0) * s.lds;
        for (int j = 0; j < ch.nc; ++j)
            for (int64_t i = 0; i < s.rows; ++i) amax = std::max(amax, std::fabs(src[i + j * s.lds]));
        return amax;
    }

    void fill(std::vector<uint8_t>& st) {
        st.assign(size_t(bytes), 0);
        // scale groups: the largest entry over all chunks of a group; row
        // groups: the largest exponent of (own scale x 2^c) over the group's
        // nonzero chunks
        int32_t ngrp = 0, nrg = 0;
        for (int32_t g : sgrp) ngrp = std::max(ngrp, g + 1);
        for (int32_t g : rgrp) nrg = std::max(nrg, g + 1);
        std::vector<double> gmax(size_t(ngrp), 0.0);
        std::vector<int> rexp(size_t(nrg), INT32_MIN);
        if (ngrp > 0 || nrg > 0) {
            std::vector<double> cmax(chunks.size(), 0.0);
            #pragma omp parallel for schedule(dynamic, 64)
            for (int64_t si = 0; si < int64_t(slabs.size()); ++si) {
                const SSlab& sl = slabs[size_t(si)];
                for (int32_t c = sl.c0; c < sl.c0 + sl.nch; ++c)
                    if (sgrp[size_t(c)] >= 0 || rgrp[size_t(c)] >= 0) cmax[size_t(c)] = chunk_amax(sl, chunks[size_t(c)]);
            }
            for (size_t c = 0; c < chunks.size(); ++c) {
                if (sgrp[c] >= 0) gmax[size_t(sgrp[c])] = std::max(gmax[size_t(sgrp[c])], cmax[c]);
                if (rgrp[c] >= 0 && cmax[c] > 0) {
                    int ex = 0;
                    std::frexp(cmax[c], &ex);   // own scale 2^(ex - 15)
                    rexp[size_t(rgrp[c])] = std::max(rexp[size_t(rgrp[c])], ex - 15 + cexp[c]);
                }
            }
        }
        #pragma omp parallel for schedule(dynamic, 64)
        for (int64_t si = 0; si < int64_t(slabs.size()); ++si) {
            const SSlab& s = slabs[size_t(si)];
            for (int32_t c = s.c0; c < s.c0 + s.nch; ++c) {
                SChunk& ch = chunks[size_t(c)];
                uint8_t* dst = st.data() + ch.byte_off;
                const double* src = s.src + s.r0 + int64_t(ch.col0) * s.lds;
                const int64_t ldc = pad_fmt(s.rows, ch.fmt);
                if (ch.fmt == FMT_F64) {
                    for (int j = 0; j < ch.nc; ++j)
                        std::memcpy(dst + size_t(j * ldc) * 8, src + j * s.lds, size_t(s.rows) * 8);
                } else if (ch.fmt == FMT_F32) {
                    for (int j = 0; j < ch.nc; ++j) {
                        float* d = reinterpret_cast<float*>(dst) + j * ldc;
                        for (int64_t i = 0; i < s.rows; ++i) d[i] = float(src[i + j * s.lds]);
                    }
                } else if (ch.fmt == FMT_I24) {
                    // power-of-two scale bringing the chunk's largest entry to
                    // [2^21, 2^22); u = v + 2^22 as 16-bit high and 8-bit low parts
                    double amax = 0;
                    for (int j = 0; j < ch.nc; ++j)
                        for (int64_t i = 0; i < s.rows; ++i) amax = std::max(amax, std::fabs(src[i + j * s.lds]));
                    int ex = 0;
                    if (amax > 0) std::frexp(amax, &ex);
                    const double scale = amax > 0 ? std::ldexp(1.0, ex - 22) : 1.0;
                    ch.scale = float(scale);
                    const double inv = 1.0 / scale;
                    for (int j = 0; j < ch.nc; ++j) {
                        uint16_t* hi = reinterpret_cast<uint16_t*>(dst + size_t(j) * size_t(ldc) * 3);
                        uint8_t* lo = dst + size_t(j) * size_t(ldc) * 3 + size_t(ldc) * 2;
                        for (int64_t i = 0; i < ldc; ++i) {   // padding rows decode to 0
                            const double q =
                                i < s.rows ? std::nearbyint(src[i + j * s.lds] * inv) : 0.0;
                            const uint32_t u = uint32_t(int32_t(std::max(-4194303.0, std::min(4194303.0, q))) + 4194304);
                            hi[i] = uint16_t(u >> 8);
                            lo[i] = uint8_t(u & 0xffu);
                        }
                    }
                } else {
                    // power-of-two scale bringing the chunk's (or its scale
                    // group's) largest entry to [2^14, 2^15); row groups: F 2^-c
                    const int32_t g = sgrp[size_t(c)], rg = rgrp[size_t(c)];
                    const double amax = g >= 0 ? gmax[size_t(g)] : chunk_amax(s, ch);
                    int ex = 0;
                    if (amax > 0) std::frexp(amax, &ex);
                    double scale = amax > 0 ? std::ldexp(1.0, ex - 15) : 1.0;
                    if (rg >= 0 && rexp[size_t(rg)] != INT32_MIN)
                        scale = std::ldexp(1.0, rexp[size_t(rg)] - cexp[size_t(c)]);
                    ch.scale = float(scale);
                    const double inv = 1.0 / scale;
                    for (int j = 0; j < ch.nc; ++j) {
                        uint16_t* d = reinterpret_cast<uint16_t*>(dst) + j * ldc;
                        if (ch.fmt == FMT_I16)   // padding rows decode to 0
                            for (int64_t i = s.rows; i < ldc; ++i) d[i] = 0x8000u;
                        for (int64_t i = 0; i < s.rows; ++i) {
                            if (ch.fmt == FMT_I16) {
                                // round to nearest, |value| < 2^15 after scaling;
                                // stored offset-binary (value + 2^15)
                                const double q = std::nearbyint(src[i + j * s.lds] * inv);
                                d[i] = uint16_t(int(std::max(-32767.0, std::min(32767.0, q))) + 32768);
                                continue;
                            }
                            const float v = float(src[i + j * s.lds] * inv);
                            d[i] = ch.fmt == FMT_F16 ? to_f16(v) : to_bf16(v);
                        }
                    }
                }
            }
        }
    }
    // FP64 stores of device-resident leaves: the copies fill() would make
    void fill_device(Plan& p) const {
        p.dev_src = true;
        p.dev_store_bytes = bytes;
        p.dev_copies.clear();
        for (const SSlab& sl : slabs)
            for (int32_t c = sl.c0; c < sl.c0 + sl.nch; ++c) {
                const SChunk& ch = chunks[size_t(c)];
                p.dev_copies.push_back(DevCopy{uint64_t(ch.byte_off), sl.src + sl.r0 + int64_t(ch.col0) * sl.lds,
                                               sl.lds, int32_t(sl.rows), int32_t(ch.nc),
                                               int32_t(pad_fmt(sl.rows, ch.fmt)), 0});
            }
    }
    int64_t slab_elem_off(int id) const {  // FP64 stores only: element offset of column 0
        return chunks[size_t(slabs[size_t(id)].c0)].byte_off / 8;
    }
};

struct TBuilder {
    TPass& P;
    std::vector<std::pair<int64_t, TUnit>> tmp[3];  // (cost, unit) per class
    explicit TBuilder(TPass& p) : P(p) {}

    // one output of `ncols` columns at `out`, fed by `slabs`
    void add(uint32_t out, int64_t ncols, const std::vector<TSlab>& slabs) {
        for (const TSlab& s : slabs) P.alg_bytes += int64_t(sizeof(double)) * s.rows * (ncols + 1);
        P.alg_bytes += int64_t(sizeof(double)) * ncols * (P.mode != OUT_SET ? 2 : 1);
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
                TUnit u{runs[0].first, runs[0].second, uint32_t(out + c0), uint16_t(c0), uint8_t(nc), TU_DIRECT};
                tmp[0].push_back({cost(u), u});
            } else {
                TGroup g{P.nslots, uint32_t(runs.size()), uint32_t(out + c0), uint32_t(nc)};
                P.groups.push_back(g);
                for (auto& r : runs) {
                    TUnit u{r.first, r.second, P.nslots++, uint16_t(c0), uint8_t(nc), 0};
                    tmp[0].push_back({cost(u), u});
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

// Reorders the reduced-precision chunks [s, e) of one tile and format into
// packs: the widest chunk is paired with the narrowest one that fits next to
// it in the format's capacity, repeatedly; the second part of a pair is
// flagged GC_PACK2 and follows its first part.
void pack_chunks(std::vector<GChunk>& ch, uint32_t s, uint32_t e) {
    if (e - s < 2 || ch[s].fmt == FMT_F64) return;
    const int cap = chunk_cols(ch[s].fmt);
    std::vector<GChunk> g(ch.begin() + s, ch.begin() + e);
    std::stable_sort(g.begin(), g.end(), [](const GChunk& a, const GChunk& b) { return a.nc > b.nc; });
    std::vector<GChunk> out;
    out.reserve(g.size());
    size_t i = 0, k = g.size();
    while (i < k) {
        out.push_back(g[i]);
        if (k - 1 > i && g[i].nc + g[k - 1].nc <= cap) {
            GChunk second = g[k - 1];
            second.flags |= GC_PACK2;
            out.push_back(second);
            --k;
        }
        ++i;
    }
    std::copy(out.begin(), out.end(), ch.begin() + s);
}

// N-form pass: one segment per output tile; the chunks of every slab that
// covers the tile.
struct NBuilder {
    NPass& P;
    const Store& S;
    bool keep_order = false;   // segments in the order built (tree sweeps), not by cost
    NBuilder(NPass& p, const Store& s) : P(p), S(s) {}
    std::vector<std::pair<int64_t, NSeg>> tmp[NFMT];
    uint32_t cb = 0;
    int64_t bytes = 0, rows = 0, alg = 0;
    void begin(int64_t tile_rows) { cb = uint32_t(P.chunks.size()); bytes = 0; rows = tile_rows; alg = 0; }
    void slab(int id, uint32_t vbase) {
        const SSlab& s = S.slabs[size_t(id)];
        for (int32_t c = s.c0; c < s.c0 + s.nch; ++c) {
            const SChunk& ch = S.chunks[size_t(c)];
            P.chunks.push_back({uint64_t(ch.byte_off), uint32_t(vbase + uint32_t(ch.col0)), uint16_t(ch.nc), ch.fmt, 0,
                                ch.scale});
            bytes += pad_fmt(s.rows, ch.fmt) * ch.nc * fmt_bytes(ch.fmt);
            alg += int64_t(ch.nc) * (rows * fmt_bytes(ch.fmt) + 8);
        }
    }
    // one segment per storage format present in the tile (OUT_SET passes,
    // which overwrite, are single-format: uniform-H is FP64 only)
    void end(uint32_t out, int64_t rows_, bool keep_empty) {
        const uint32_t ce = uint32_t(P.chunks.size());
        if (ce == cb && !keep_empty) return;
        std::stable_sort(P.chunks.begin() + cb, P.chunks.end(),
                         [](const GChunk& a, const GChunk& b) { return a.fmt < b.fmt; });
        if (ce == cb) tmp[FMT_F64].push_back({0, NSeg{cb, ce, out, uint16_t(rows_), uint16_t(pad_rows(rows_))}});
        for (uint32_t s = cb; s < ce;) {
            const uint8_t f = P.chunks[s].fmt;
            uint32_t e = s;
            int64_t by = 0;
            for (; e < ce && P.chunks[e].fmt == f; ++e) by += pad_fmt(rows_, f) * P.chunks[e].nc * fmt_bytes(f);
            pack_chunks(P.chunks, s, e);
            tmp[f].push_back({by, NSeg{s, e, out, uint16_t(rows_), uint16_t(pad_fmt(rows_, f))}});
            s = e;
        }
        P.alg_bytes += alg + int64_t(sizeof(double)) * rows_ * (P.mode != OUT_SET ? 2 : 1);
    }
    void finish() {
        for (int f = 0; f < NFMT; ++f) {
            if (!keep_order)
                std::stable_sort(tmp[f].begin(), tmp[f].end(),
                                 [](const auto& a, const auto& b) { return a.first > b.first; });
            P.segs[f].clear();
            for (auto& e : tmp[f]) {
                P.segs[f].push_back(e.second);
                P.bytes += e.first;
            }
        }
    }
};

// Tile T-form pass: objects (low-rank blocks / cluster bases / column tiles
// of the near field) own an output of `ncols` values and receive one slab per
// input tile.  Objects fed by one slab write their chunks' results directly;
// objects fed by several write per-slab partials that a finish pass sums in
// slab order.
// Plan-level choices of the running planner call (hlrc_options), read by the
// builders; set for the duration of a plan_* call by KnobScope.
struct PlanKnobs {
    uint32_t finish_slots = FINISH_SLOTS;
    int piece_tiles = WT_MAXT;
    int near_field = 0;            // hlrc_options.near_field (0: the default, 2)
    // the near field on a side stream (every kind of plan: 0 H, 1 uniform-H,
    // 2 H^2), unless the caller asks for it fused
    bool side_dense(int /*kind*/) const { return near_field != 1; }
};
thread_local PlanKnobs g_knobs;
struct KnobScope {
    PlanKnobs saved;
    explicit KnobScope(const hlrc_options& o) : saved(g_knobs) {
        g_knobs.finish_slots = o.finish_slots > 0 ? uint32_t(o.finish_slots) : FINISH_SLOTS;
        g_knobs.piece_tiles = o.piece_tiles > 0 ? o.piece_tiles : WT_MAXT;
        g_knobs.near_field = o.near_field;
    }
    ~KnobScope() { g_knobs = saved; }
};
hlrc_status check_knobs(const hlrc_options& o) {
    if (o.finish_slots != 0 && (o.finish_slots < 2 || o.finish_slots > 64))
        return fail(HLRC_ERR_ARG, "finish_slots %d outside 2..64", o.finish_slots);
    if (o.piece_tiles != 0 && (o.piece_tiles < 1 || o.piece_tiles > WT_MAXT))
        return fail(HLRC_ERR_ARG, "piece_tiles %d outside 1..%d", o.piece_tiles, WT_MAXT);
    if (o.near_field < 0 || o.near_field > 2)
        return fail(HLRC_ERR_ARG, "near_field %d outside 0..2", o.near_field);
    if (o.leaves_on_device != 0 && o.leaves_on_device != 1)
        return fail(HLRC_ERR_ARG, "leaves_on_device must be 0 or 1 (got %d)", o.leaves_on_device);
    return HLRC_OK;
}

struct TTBuilder {
    TTPass& P;
    const Store& S;
    std::vector<std::pair<int64_t, TTSeg>> tmp[NFMT];
    std::vector<int64_t> pbase, ncol;
    std::vector<uint32_t> oout;
    uint32_t cb = 0, voff = 0;
    int64_t bytes = 0, rows = 0;
    TTBuilder(TTPass& p, const Store& s, size_t nobj) : P(p), S(s), pbase(nobj, -2), ncol(nobj, 0), oout(nobj, 0) {}

    void object(size_t id, uint32_t out, int64_t ncols, int64_t nslabs) {
        ncol[id] = ncols;
        oout[id] = out;
        if (nslabs > 1) {
            pbase[id] = P.npart;
            P.groups.push_back({uint32_t(P.npart), uint32_t(nslabs), out, uint32_t(ncols)});
            P.npart += nslabs * ncols;
        } else {
            pbase[id] = -1;
        }
        P.alg_bytes += int64_t(sizeof(double)) * ncols * (P.mode != OUT_SET ? 2 : 1);
    }
    void begin(int64_t v_off, int64_t tile_rows) {
        cb = uint32_t(P.chunks.size());
        voff = uint32_t(v_off);
        rows = tile_rows;
        bytes = 0;
    }
    // columns [lo, lo + ncol[id]) of slab `sid` feed object `id` as its slab number `k`
    void slab(int sid, size_t id, int64_t k, int64_t lo = 0) {
        const SSlab& s = S.slabs[size_t(sid)];
        const int64_t hi = lo + ncol[id];
        for (int32_t c = s.c0; c < s.c0 + s.nch; ++c) {
            const SChunk& ch = S.chunks[size_t(c)];
            if (ch.col0 < lo || ch.col0 >= hi) continue;
            const int64_t j = ch.col0 - lo;
            GChunk g{uint64_t(ch.byte_off), 0, uint16_t(ch.nc), ch.fmt, 0, ch.scale};
            if (pbase[id] < 0) { g.vo = uint32_t(oout[id] + j); g.flags = TT_DIRECT; }
            else g.vo = uint32_t(pbase[id] + k * ncol[id] + j);
            P.chunks.push_back(g);
            bytes += pad_fmt(s.rows, ch.fmt) * ch.nc * fmt_bytes(ch.fmt);
            P.alg_bytes += rows * ch.nc * fmt_bytes(ch.fmt);
        }
    }
    void end() {
        const uint32_t ce = uint32_t(P.chunks.size());
        if (ce == cb) return;
        std::stable_sort(P.chunks.begin() + cb, P.chunks.end(),
                         [](const GChunk& a, const GChunk& b) { return a.fmt < b.fmt; });
        for (uint32_t s = cb; s < ce;) {
            const uint8_t f = P.chunks[s].fmt;
            uint32_t e = s;
            int64_t by = 0;
            for (; e < ce && P.chunks[e].fmt == f; ++e) by += pad_fmt(rows, f) * P.chunks[e].nc * fmt_bytes(f);
            pack_chunks(P.chunks, s, e);
            tmp[f].push_back({by, TTSeg{s, e, voff, uint16_t(rows), uint16_t(pad_fmt(rows, f))}});
            s = e;
        }
        P.alg_bytes += int64_t(sizeof(double)) * rows;
    }
    void finish() {
        for (int f = 0; f < NFMT; ++f) {
            std::stable_sort(tmp[f].begin(), tmp[f].end(), [](const auto& a, const auto& b) { return a.first > b.first; });
            P.segs[f].clear();
            for (auto& e : tmp[f]) {
                P.segs[f].push_back(e.second);
                P.bytes += e.first;
            }
        }
        // Outputs with more than FINISH_SLOTS tiles are summed in two levels,
        // so that no warp adds more than FINISH_SLOTS slots in a row: the
        // slots are cut into runs whose sums go to a scratch region appended
        // to the partial array (layout [run][column], like the slots), and
        // the output's group then sums the runs.  The order of all additions
        // depends on the shapes only.
        for (TGroup& g : P.groups) {
            const uint32_t FS = g_knobs.finish_slots;
            if (g.nslots <= FS) continue;
            const uint32_t nrun = (g.nslots + FS - 1) / FS;
            const uint32_t scratch = uint32_t(P.npart);
            for (uint32_t r = 0; r < nrun; ++r) {
                const uint32_t s0 = r * FS;
                P.groups1.push_back({g.slot0 + s0 * g.nc, std::min(FS, g.nslots - s0), scratch + r * g.nc, g.nc});
            }
            P.npart += int64_t(nrun) * g.nc;
            g.slot0 = scratch;
            g.nslots = nrun;
        }
    }
};

inline double flops_gemv(double m, double n) { return 2.0 * m * n + 2.0 * m; }

// Transposed near field y_sigma += alpha sum D^T x as a tile T-form pass:
// CTAs run over row tiles, objects are the column tiles, and every (dense
// block, row tile) slab that covers a column tile is one of its inputs.
template <typename DenseOf>
void plan_dense_transposed(TTPass& P, const Store& st, const Tiles& tr, const Tiles& tc,
                           const std::vector<std::vector<int64_t>>& dense_by_rowtile,
                           const std::vector<std::vector<int>>& dslab, DenseOf dense) {
    P.in = V_X; P.out = V_Y; P.mode = OUT_ADD_ALPHA;
    TTBuilder tb(P, st, size_t(tc.n()));
    std::vector<int64_t> cnt(size_t(tc.n()), 0);
    for (int64_t t = 0; t < tr.n(); ++t)
        for (int64_t i : dense_by_rowtile[size_t(t)]) {
            int64_t col0, ncols;
            dense(i, col0, ncols);
            for (int64_t s = tc.first(col0); s < tc.first(col0 + ncols); ++s) ++cnt[size_t(s)];
        }
    for (int64_t s = 0; s < tc.n(); ++s)
        if (cnt[size_t(s)] > 0) tb.object(size_t(s), uint32_t(tc.lo(s)), tc.size(s), cnt[size_t(s)]);
    std::vector<int64_t> k(size_t(tc.n()), 0);
    std::vector<size_t> pos(dslab.size(), 0);
    for (int64_t t = 0; t < tr.n(); ++t) {
        tb.begin(tr.lo(t), tr.size(t));
        for (int64_t i : dense_by_rowtile[size_t(t)]) {
            int64_t col0, ncols;
            dense(i, col0, ncols);
            const int sid = dslab[size_t(i)][pos[size_t(i)]++];
            for (int64_t s = tc.first(col0); s < tc.first(col0 + ncols); ++s)
                tb.slab(sid, size_t(s), k[size_t(s)]++, tc.lo(s) - col0);
        }
        tb.end();
    }
    tb.finish();
}

// column tile boundaries inside [col0, col0+ncols), relative to col0
std::vector<int64_t> inner_cuts(const Tiles& tc, int64_t col0, int64_t ncols) {
    std::vector<int64_t> c;
    for (int64_t s = tc.first(col0) + 1; s < tc.first(col0 + ncols); ++s) c.push_back(tc.lo(s) - col0);
    return c;
}

// VALR column precisions (compress/valr.hh:402-510): delta = eps sigma_0,
// tol from  Sigma_l 1/sigma_l tol^2 - tol + delta = 0 (smaller root),
// u_l = tol / sigma_l; a column may use the cheapest format whose unit
// roundoff is <= u_l.  Reduced-precision stores hold FP32 and FP16 only:
// columns whose u_l asks for more than FP32 (possible when the block's
// singular values span many orders of magnitude and the quadratic's root is
// clamped) are stored in FP32.
void valr_formats(const double* sv, int64_t k, double eps, uint8_t* fmt, int prec) {
    if (k <= 0) return;
    const double delta = eps * sv[0];
    double sum = 0;
    for (int64_t l = 0; l < k; ++l) sum += sv[l] > 0 ? 1.0 / sv[l] : 0.0;
    double tol = delta;
    if (sum > 0) {
        const double p = 1.0 / sum, q = delta / sum;
        const double t = std::max(0.0, p * p / 4 - q);
        tol = std::min(std::fabs(p / 2 + std::sqrt(t)), std::fabs(p / 2 - std::sqrt(t)));
    }
    for (int64_t l = 0; l < k; ++l) {
        const double u = sv[l] > 0 ? tol / sv[l] : 1.0;
        // MIXED: FP16 (unit roundoff 2^-11) where it suffices.  BFP: the
        // column's bit rate ceil(-log2 u) (bfp.hh:79-80) fits a 16-bit
        // integer mantissa scaled to [2^14, 2^15), whose rounding error is
        // at most 2^-15 of the chunk's largest entry; other columns take 24
        // bits (scaled to [2^21, 2^22): 2^-22)
        if (prec == HLRC_PREC_BFP) fmt[l] = u >= 0x1.0p-15 ? FMT_I16 : FMT_I24;
        else fmt[l] = u >= 0x1.0p-11 ? FMT_F16 : FMT_F32;
    }
}

// Checks every descriptor of the N-form and tile-T-form passes against the
// store, the vector lengths and the alignment the kernels rely on (16-byte
// chunk starts; columns of pad_fmt(rows, fmt) elements; lane pairs inside
// the padded column).  A violation is a planner bug: the upload is refused
// instead of handing the GPU an out-of-bounds address.
hlrc_status validate_plan(const Plan& p) {
    const int64_t store = p.store_size();
    auto vec_len = [&](int name) -> int64_t {
        switch (name) {
            case V_X: return std::max(p.nrows, p.ncols);
            case V_Y: return std::max(p.nrows, p.ncols);
            case V_T: return p.n_t;
            default: return p.n_t2;
        }
    };
    // reduced-precision segments must be one contiguous run of columns in
    // the store (the multi-RHS kernels stream them as such)
    auto contiguous = [&](const std::vector<GChunk>& ch, uint32_t cb, uint32_t ce, int f, int64_t ld) -> bool {
        if (f == FMT_F64 || ce <= cb) return true;
        std::vector<uint64_t> offs;
        offs.reserve(ce - cb);
        for (uint32_t c = cb; c < ce; ++c) offs.push_back(ch[c].byte_off);
        std::vector<uint32_t> idx(ce - cb);
        for (uint32_t k = 0; k < idx.size(); ++k) idx[k] = k;
        std::sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t b) { return offs[a] < offs[b]; });
        uint64_t expect = offs[idx[0]];
        for (uint32_t k : idx) {
            if (offs[k] != expect) return false;
            expect += uint64_t(ld) * fmt_bytes(f) * ch[cb + k].nc;
        }
        return true;
    };
    auto chunk_ok = [&](const GChunk& c, int64_t rows) -> bool {
        if (c.nc == 0 || rows <= 0 || rows > TILE) return false;
        if (c.byte_off % 16 != 0) return false;
        const int64_t ld = pad_fmt(rows, c.fmt);
        return int64_t(c.byte_off) + ld * c.nc * fmt_bytes(c.fmt) <= store;
    };
    for (size_t pi = 0; pi < p.npasses.size(); ++pi) {
        const NPass& np = p.npasses[pi];
        for (int f = 0; f < NFMT; ++f)
            for (const NSeg& s : np.segs[f]) {
                if (s.ld != pad_fmt(s.rows, f) || s.ce < s.cb || s.ce > np.chunks.size())
                    return fail(HLRC_ERR_INTERNAL, "N-pass %zu: bad segment", pi);
                if (!contiguous(np.chunks, s.cb, s.ce, f, s.ld))
                    return fail(HLRC_ERR_INTERNAL, "N-pass %zu: segment is not one column run", pi);
                if (int64_t(s.out) + s.rows > vec_len(np.out))
                    return fail(HLRC_ERR_INTERNAL, "N-pass %zu: output tile outside the vector", pi);
                for (uint32_t c = s.cb; c < s.ce; ++c) {
                    const GChunk& g = np.chunks[c];
                    if (g.fmt != f || !chunk_ok(g, s.rows))
                        return fail(HLRC_ERR_INTERNAL, "N-pass %zu: chunk %u outside the store or misaligned", pi, c);
                    const bool t = (g.vo & VEC_T) != 0;
                    if (int64_t(g.vo & ~VEC_T) + g.nc > vec_len(t ? np.vt : np.vx))
                        return fail(HLRC_ERR_INTERNAL, "N-pass %zu: chunk %u vector outside its array", pi, c);
                }
            }
        // tree sweeps: FP64 segments whose chunks follow one another, levels
        // and subtrees that partition them, rank runs that partition each
        // level, stage and mirror entries inside the shared memory (16-byte
        // aligned stage runs)
        if (np.cta_begin.empty() && np.tree_level.empty()) continue;
        const std::vector<NSeg>& sg = np.segs[FMT_F64];
        const std::vector<int32_t>&cb = np.cta_begin, &tl = np.tree_level;
        constexpr int TC = TREE_CLUSTER;
        const size_t nsub = cb.size() - 1;
        bool ok = cb.size() >= 2 && tl.size() >= 2 && cb.front() == 0 && tl.front() == 0 &&
                  cb.back() == int32_t(tl.size()) - 1 && tl.back() == int32_t(sg.size()) && !sg.empty() &&
                  sg.back().ce == np.chunks.size() && np.tree_seg.size() == sg.size() &&
                  np.tree_part.size() == (tl.size() - 1) * (TC + 1) && np.tree_chunk.size() == np.chunks.size() &&
                  np.tree_cta_ext.size() == nsub + 1 && np.tree_cta_ext.front() == 0 &&
                  np.tree_cta_ext.back() == int32_t(np.tree_ext.size()) &&
                  tree_smem_bytes(np.tree_stage, np.tree_mirror, np.tree_levels, np.tree_segs, np.tree_chunks,
                                  np.tree_items) <= TREE_SMEM &&
                  np.tree_stage % 2 == 0 && (np.vt == np.out) && (np.mode == OUT_SET || np.mode == OUT_ADD) &&
                  nsub * TC < (size_t(1) << 31);
        for (int f = 0; f < NFMT && ok; ++f) ok = f == FMT_F64 || np.segs[f].empty();
        for (size_t i = 1; i < cb.size() && ok; ++i) ok = cb[i] > cb[i - 1];
        for (size_t i = 1; i < tl.size() && ok; ++i) ok = tl[i] > tl[i - 1];
        for (size_t i = 1; i < np.tree_cta_ext.size() && ok; ++i) ok = np.tree_cta_ext[i] >= np.tree_cta_ext[i - 1];
        for (size_t s = 0; s < sg.size() && ok; ++s) ok = sg[s].cb == (s ? sg[s - 1].ce : 0u);
        for (size_t b = 0; b < nsub && ok; ++b) {
            const int32_t s0 = tl[size_t(cb[b])], s1 = tl[size_t(cb[b + 1])];
            ok = cb[b + 1] - cb[b] <= np.tree_levels && s1 - s0 <= np.tree_segs &&
                 int64_t(sg[size_t(s1 - 1)].ce) - int64_t(sg[size_t(s0)].cb) <= np.tree_chunks;
            for (int32_t g = cb[b]; g < cb[b + 1] && ok; ++g) {
                const int32_t* part = &np.tree_part[size_t(g) * (TC + 1)];
                ok = part[0] == tl[size_t(g)] && part[TC] == tl[size_t(g) + 1];
                for (int r = 0; r < TC && ok; ++r) {
                    ok = part[r + 1] >= part[r];
                    int64_t items = 0, stage_end = 0;
                    for (int32_t q = part[r]; q < part[r + 1] && ok; ++q)
                        for (uint32_t c = sg[size_t(q)].cb; c < sg[size_t(q)].ce && ok; ++c) {
                            ++items;
                            const TreeChunk& t = np.tree_chunk[c];
                            stage_end = int64_t(t.stage) + int64_t(np.chunks[c].nc) * sg[size_t(q)].ld;
                            ok = t.stage % 2 == 0 && stage_end <= np.tree_stage &&
                                 int64_t(t.mirror) + np.chunks[c].nc <= np.tree_mirror;
                        }
                    ok = ok && items <= np.tree_items;
                }
            }
            for (int32_t q = s0; q < s1 && ok; ++q)
                ok = np.tree_seg[size_t(q)] >= 0 && np.tree_seg[size_t(q)] + sg[size_t(q)].rows <= np.tree_mirror;
            for (int32_t e = np.tree_cta_ext[b]; e < np.tree_cta_ext[b + 1] && ok; ++e) {
                const TreeExt& x = np.tree_ext[size_t(e)];
                const bool t = (x.v_off & VEC_T) != 0;
                ok = int64_t(x.mirror) < np.tree_mirror && int64_t(x.v_off & ~VEC_T) < vec_len(t ? np.vt : np.vx);
            }
        }
        if (!ok) return fail(HLRC_ERR_INTERNAL, "N-pass %zu: malformed tree sweep", pi);
    }
    for (size_t pi = 0; pi < p.ttpasses.size(); ++pi) {
        const TTPass& tp = p.ttpasses[pi];
        for (int f = 0; f < NFMT; ++f)
            for (const TTSeg& s : tp.segs[f]) {
                if (s.ld != pad_fmt(s.rows, f) || s.ce < s.cb || s.ce > tp.chunks.size())
                    return fail(HLRC_ERR_INTERNAL, "T-pass %zu: bad segment", pi);
                if (!contiguous(tp.chunks, s.cb, s.ce, f, s.ld))
                    return fail(HLRC_ERR_INTERNAL, "T-pass %zu: segment is not one column run", pi);
                if (int64_t(s.v_off) + s.rows > vec_len(tp.in))
                    return fail(HLRC_ERR_INTERNAL, "T-pass %zu: input tile outside the vector", pi);
                for (uint32_t c = s.cb; c < s.ce; ++c) {
                    const GChunk& g = tp.chunks[c];
                    if (g.fmt != f || !chunk_ok(g, s.rows))
                        return fail(HLRC_ERR_INTERNAL, "T-pass %zu: chunk %u outside the store or misaligned", pi, c);
                    const int64_t lim = (g.flags & TT_DIRECT) ? vec_len(tp.out) : tp.npart;
                    if (int64_t(g.vo) + g.nc > lim)
                        return fail(HLRC_ERR_INTERNAL, "T-pass %zu: chunk %u output outside its array", pi, c);
                }
            }
        for (const TGroup& g : tp.groups)
            if (int64_t(g.slot0) + int64_t(g.nslots) * g.nc > tp.npart || int64_t(g.out) + g.nc > vec_len(tp.out))
                return fail(HLRC_ERR_INTERNAL, "T-pass %zu: finish group outside its arrays", pi);
        for (const TGroup& g : tp.groups1)
            if (int64_t(g.slot0) + int64_t(g.nslots) * g.nc > tp.npart || int64_t(g.out) + g.nc > tp.npart)
                return fail(HLRC_ERR_INTERNAL, "T-pass %zu: first-level finish group outside the partials", pi);
    }
    // side stages lead their list and are plain N-form passes adding into y
    // from x and the store only: they run beside the stages after them
    for (int op = 0; op < 3; ++op) {
        bool main_seen = false;
        for (const Stage& sg : p.stages_nf[op]) {
            if (!sg.side) { main_seen = true; continue; }
            if (main_seen || sg.kind != 1 || sg.idx < 0 || size_t(sg.idx) >= p.npasses.size())
                return fail(HLRC_ERR_INTERNAL, "op %d: side stage out of place", op);
            const NPass& np = p.npasses[size_t(sg.idx)];
            if (np.out != V_Y || np.mode != OUT_ADD_ALPHA || !np.cta_begin.empty())
                return fail(HLRC_ERR_INTERNAL, "op %d: side stage is not a plain pass into y", op);
            for (const GChunk& g : np.chunks)
                if (g.vo & VEC_T) return fail(HLRC_ERR_INTERNAL, "op %d: side stage reads coefficients", op);
        }
    }
    return HLRC_OK;
}

uint8_t default_format(int prec) {
    switch (prec) {
        case HLRC_PREC_F32: return FMT_F32;
        case HLRC_PREC_BF16: return FMT_BF16;
        case HLRC_PREC_F16: return FMT_F16;
        default: return FMT_F64;
    }
}

}  // namespace

// --------------------------------------------------------------------- H
// The 64-vector product of a 16-bit H store, op N (WidePlan): units of the
// column-cluster T-form and the static exponents of t.  Low-rank blocks are
// grouped by their column index set (blocks of one group read the same x
// rows); a group's columns are stacked in units of at most WT_MAXN (a block
// of higher rank is cut into slices), and a group spanning more than
// WT_MAXT tiles is cut into pieces, each writing FP32 partials that a finish
// group per block sums in piece order.
hlrc_status plan_wide(const hlrc_h_desc& d, const Tiles& tc, const std::vector<int64_t>& toff,
                      const std::vector<int32_t>& cblk, const std::vector<std::vector<int>>& slabV, const Store& st,
                      Plan& p) {
    WidePlan& W = p.wide;
    W = WidePlan();
    for (int64_t t = 0; t < tc.n(); ++t)
        W.tiles.push_back(WTTile{uint32_t(tc.lo(t)), uint16_t(tc.size(t)), uint16_t(pad_fmt(tc.size(t), FMT_F16))});
    W.t_exp.assign(size_t(std::max<int64_t>(1, p.n_t)), 0);
    std::map<std::pair<int64_t, int64_t>, std::vector<int64_t>> groups;   // (col0, ncols) -> blocks
    for (int64_t i = 0; i < d.nblocks; ++i) {
        const hlrc_block& b = d.blocks[i];
        if (toff[size_t(i)] < 0) continue;
        for (int64_t l = 0; l < b.rank; ++l) W.t_exp[size_t(toff[size_t(i)] + l)] = int8_t(cblk[size_t(i)]);
        groups[{b.col0, b.ncols}].push_back(i);
    }
    struct Item { int64_t blk, l0, k; };
    auto slab_a16 = [&](int64_t i, int64_t ti, int64_t l0) -> uint64_t {
        const SSlab& sl = st.slabs[size_t(slabV[size_t(i)][size_t(ti)])];
        const uint64_t off = uint64_t(st.chunks[size_t(sl.c0)].byte_off) + uint64_t(l0) * uint64_t(pad_fmt(sl.rows, FMT_F16)) * 2;
        return off / 16;
    };
    std::vector<std::pair<int64_t, size_t>> cost;   // (cost, unit index) for the order
    for (const auto& kv : groups) {
        const int64_t col0 = kv.first.first, ncols = kv.first.second;
        const int64_t t0 = tc.first(col0), T = tc.first(col0 + ncols) - t0;
        std::vector<Item> items;
        for (int64_t i : kv.second)
            for (int64_t l0 = 0; l0 < d.blocks[i].rank; l0 += WT_MAXN)
                items.push_back({i, l0, std::min<int64_t>(WT_MAXN, d.blocks[i].rank - l0)});
        size_t a = 0;
        while (a < items.size()) {   // one subset: items [a, e) with at most WT_MAXN columns
            size_t e = a;
            int64_t nc = 0;
            // stacked columns start on multiples of 8 (8-column TMA boxes)
            while (e < items.size() && nc + (items[e].k + 7) / 8 * 8 <= WT_MAXN && int(e - a) < WT_MAXB)
                nc += (items[e++].k + 7) / 8 * 8;
            const int64_t PT = g_knobs.piece_tiles;
            const int64_t P = (T + PT - 1) / PT;
            const int64_t part0 = P > 1 ? W.npart : 0;
            if (P > 1) W.npart += P * nc;
            for (int64_t q = 0; q < P; ++q) {
                const int64_t q0 = t0 + (T * q) / P, q1 = t0 + (T * (q + 1)) / P;
                WTUnit u{};
                u.tile0 = uint32_t(q0);
                u.ntiles = uint16_t(q1 - q0);
                u.ncols = uint16_t(nc);
                u.blk0 = uint32_t(W.blks.size());
                u.slab0 = uint32_t(W.slabs.size());
                u.nblk = uint16_t(e - a);
                u.piece = uint16_t(q);
                u.npieces = uint16_t(P);
                u.part0 = uint32_t(part0);
                int64_t off = 0;
                for (size_t j = a; j < e; ++j) {
                    const Item& it = items[j];
                    const SSlab& s0 = st.slabs[size_t(slabV[size_t(it.blk)][0])];
                    WTBlk wb{};
                    wb.toff = uint32_t(toff[size_t(it.blk)] + it.l0);
                    wb.k = uint16_t(it.k);
                    wb.off = uint16_t(off);
                    wb.scale = st.chunks[size_t(s0.c0)].scale;
                    wb.pbase = uint32_t(part0 + P * off);
                    W.blks.push_back(wb);
                    off += (it.k + 7) / 8 * 8;
                }
                for (int64_t t = q0; t < q1; ++t)
                    for (size_t j = a; j < e; ++j) {
                        const Item& it = items[j];
                        const uint64_t a16 = slab_a16(it.blk, t - tc.first(d.blocks[it.blk].col0), it.l0);
                        if (a16 >= (uint64_t(1) << 32)) return fail(HLRC_ERR_SHAPE, "store offset beyond 2^36 bytes");
                        W.slabs.push_back(uint32_t(a16));
                    }
                cost.push_back({(q1 - q0) * (16384 + nc * 128), W.units.size()});
                W.units.push_back(u);
            }
            if (P > 1)
                for (size_t j = a; j < e; ++j) {
                    const WTBlk& wb = W.blks[W.blks.size() - (e - j)];
                    W.groups.push_back(TGroup{wb.pbase, uint32_t(P), wb.toff, wb.k});
                }
            a = e;
        }
    }
    if (W.npart >= (int64_t(1) << 32) || W.slabs.size() >= (size_t(1) << 32))
        return fail(HLRC_ERR_SHAPE, "64-vector tables exceed 2^32 entries");
    std::stable_sort(cost.begin(), cost.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
    std::vector<WTUnit> sorted;
    sorted.reserve(W.units.size());
    for (const auto& c : cost) sorted.push_back(W.units[c.second]);
    W.units.swap(sorted);
    // every V column a unit stages lies inside the store
    for (const WTUnit& u : W.units)
        for (int t = 0; t < u.ntiles; ++t)
            for (int j = 0; j < u.nblk; ++j) {
                const uint64_t a16 = W.slabs[size_t(u.slab0) + size_t(t) * u.nblk + size_t(j)];
                const uint64_t end = a16 * 16 + uint64_t(W.blks[size_t(u.blk0) + size_t(j)].k) *
                                                     uint64_t(W.tiles[size_t(u.tile0) + size_t(t)].ld) * 2;
                if (a16 * 16 % 16 != 0 || end > uint64_t(p.store_size()))
                    return fail(HLRC_ERR_INTERNAL, "64-vector unit reads outside the store");
            }
    return HLRC_OK;
}

hlrc_status plan_h(const hlrc_h_desc& d, const hlrc_options& o, Plan& p, double expected_area) {
    if (hlrc_status ks = check_knobs(o); ks != HLRC_OK) return ks;
    const KnobScope knobs(o);
    // leaf data in device memory is never read here: FP64 stores become
    // device copies (Store::fill_device), other precisions are planned from
    // a host copy of the leaves (hlrc_upload_h)
    if (o.leaves_on_device && o.precision != HLRC_PREC_F64)
        return fail(HLRC_ERR_INTERNAL, "device-resident leaves reach the planner with an FP64 store only");
    if (d.nrows < 0 || d.ncols < 0 || d.nblocks < 0) return fail(HLRC_ERR_SHAPE, "negative matrix size");
    if (d.nblocks > 0 && !d.blocks) return fail(HLRC_ERR_ARG, "blocks == NULL");
    if (d.nrows >= (int64_t(1) << 31) || d.ncols >= (int64_t(1) << 31))
        return fail(HLRC_ERR_SHAPE, "matrix dimension exceeds 2^31-1");
    if (o.precision < HLRC_PREC_F64 || o.precision > HLRC_PREC_BFP)
        return fail(HLRC_ERR_ARG, "unknown precision %d", o.precision);
    const bool valr = o.precision == HLRC_PREC_MIXED || o.precision == HLRC_PREC_BFP;
    if (valr && !(o.mixed_eps > 0))
        return fail(HLRC_ERR_ARG, "HLRC_PREC_MIXED / HLRC_PREC_BFP need mixed_eps > 0");
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
    const double want = expected_area >= 0 ? expected_area : double(d.nrows) * double(d.ncols);
    if (area != want)
        return fail(HLRC_ERR_SHAPE, "leaf blocks cover %.0f entries, matrix has %.0f (gap or overlap)", area, want);
    const Tiles tr = make_tiles(d.nrows, rcuts), tc = make_tiles(d.ncols, ccuts);
    p.n_row_tiles = tr.n();
    p.n_col_tiles = tc.n();

    // coefficient offsets and per-tile block lists (block order preserved)
    std::vector<int64_t> toff(static_cast<size_t>(nb), -1);
    int64_t nt = 0;
    std::vector<std::vector<int64_t>> rowlist(static_cast<size_t>(tr.n())), collist(static_cast<size_t>(tc.n())),
        dense_rows(static_cast<size_t>(tr.n()));
    for (int64_t i = 0; i < nb; ++i) {
        const hlrc_block& b = d.blocks[i];
        if (b.nrows == 0 || b.ncols == 0) continue;
        const bool lr = b.kind == HLRC_LEAF_LOWRANK;
        if (lr && b.rank == 0) continue;
        if (lr) { toff[size_t(i)] = nt; nt += b.rank; }
        for (int64_t t = tr.first(b.row0); t < tr.first(b.row0 + b.nrows); ++t) {
            rowlist[size_t(t)].push_back(i);
            if (!lr) dense_rows[size_t(t)].push_back(i);
        }
        for (int64_t t = tc.first(b.col0); t < tc.first(b.col0 + b.ncols); ++t) collist[size_t(t)].push_back(i);
    }
    if (nt >= (int64_t(1) << 31)) return fail(HLRC_ERR_SHAPE, "sum of ranks exceeds 2^31-1");
    p.n_t = nt;

    // storage formats
    const uint8_t deffmt = default_format(o.precision);
    const uint8_t densefmt =
        o.precision == HLRC_PREC_BFP ? uint8_t(FMT_I24) : (valr ? uint8_t(FMT_F32) : deffmt);
    std::vector<std::vector<uint8_t>> colfmt(static_cast<size_t>(nb));
    if (valr) {
        for (int64_t i = 0; i < nb; ++i) {
            const hlrc_block& b = d.blocks[i];
            if (toff[size_t(i)] < 0) continue;
            std::vector<double> sv(static_cast<size_t>(b.rank));
            for (int64_t l = 0; l < b.rank; ++l) {
                if (b.sv) { sv[size_t(l)] = b.sv[l]; continue; }
                double nu = 0, nv = 0;
                for (int64_t r = 0; r < b.nrows; ++r) nu += b.U[r + l * b.ldu] * b.U[r + l * b.ldu];
                for (int64_t r = 0; r < b.ncols; ++r) nv += b.V[r + l * b.ldv] * b.V[r + l * b.ldv];
                sv[size_t(l)] = std::sqrt(nu * nv);
            }
            // VALR expects descending singular values; sort a copy for the
            // tolerance and map formats back to the stored column order
            std::vector<int64_t> ord(static_cast<size_t>(b.rank));
            std::iota(ord.begin(), ord.end(), 0);
            std::stable_sort(ord.begin(), ord.end(), [&](int64_t a, int64_t c) { return sv[size_t(a)] > sv[size_t(c)]; });
            std::vector<double> svs(static_cast<size_t>(b.rank));
            for (int64_t l = 0; l < b.rank; ++l) svs[size_t(l)] = sv[size_t(ord[size_t(l)])];
            std::vector<uint8_t> fs(static_cast<size_t>(b.rank));
            valr_formats(svs.data(), b.rank, o.mixed_eps, fs.data(), o.precision);
            colfmt[size_t(i)].assign(static_cast<size_t>(b.rank), FMT_F32);
            for (int64_t l = 0; l < b.rank; ++l) colfmt[size_t(i)][size_t(ord[size_t(l)])] = fs[size_t(l)];
        }
    }
    auto cf = [&](int64_t i) -> const uint8_t* { return colfmt[size_t(i)].empty() ? nullptr : colfmt[size_t(i)].data(); };

    // storage: row region (per row tile: D and U slabs), then the V region
    // ordered by column tile, so that each pass streams one contiguous
    // range per tile
    Store st;
    // 16-bit stores also serve the 64-vector product (plan_wide): the chunks
    // of a row tile form a row group with exponent c_b for the U slabs of
    // block b (2^c_b > ||V(:,l)||_1 for all l), so that the tile's run needs
    // no per-column factors, and 16-bit groups start on 128-byte boundaries
    const bool wide16 = o.precision == HLRC_PREC_F16 || o.precision == HLRC_PREC_BF16;
    std::vector<int32_t> cblk(static_cast<size_t>(nb), 0);
    if (wide16) {
        st.align128 = true;
        for (int64_t i = 0; i < nb; ++i) {
            const hlrc_block& b = d.blocks[i];
            if (toff[size_t(i)] < 0) continue;
            int c = INT32_MIN;
            for (int64_t l = 0; l < b.rank; ++l) {
                double s1 = 0;
                for (int64_t r = 0; r < b.ncols; ++r) s1 += std::fabs(b.V[r + l * b.ldv]);
                if (s1 > 0) c = std::max(c, std::ilogb(s1) + 1);
            }
            cblk[size_t(i)] = c == INT32_MIN ? 0 : std::max(-120, std::min(120, c));
        }
    }
    std::vector<std::vector<int>> slabA(static_cast<size_t>(nb)), slabV(static_cast<size_t>(nb));
    for (int64_t t = 0; t < tr.n(); ++t) {
        const int32_t rg = wide16 ? int32_t(t) : -1;
        for (int64_t i : rowlist[size_t(t)]) {
            const hlrc_block& b = d.blocks[i];
            const int64_t r0 = tr.lo(t) - b.row0, rows = tr.size(t);
            if (b.kind == HLRC_LEAF_DENSE) {
                const std::vector<int64_t> cuts = inner_cuts(tc, b.col0, b.ncols);
                slabA[size_t(i)].push_back(st.alloc(b.D, b.ldd, r0, rows, b.ncols, nullptr, densefmt, &cuts, 0, -1, rg, 0));
            } else {
                slabA[size_t(i)].push_back(st.alloc(b.U, b.ldu, r0, rows, b.rank, cf(i), deffmt, nullptr, 1, -1, rg,
                                                    cblk[size_t(i)]));
            }
        }
        st.close_region();
    }
    // 16-bit stores: the V chunks of one block share one scale over all its
    // column tiles, so the 64-vector T-form can sum a block's tiles in one
    // accumulator (the per-element precision of a 16-bit float does not
    // depend on the scale)
    for (int64_t t = 0; t < tc.n(); ++t) {
        for (int64_t i : collist[size_t(t)]) {
            const hlrc_block& b = d.blocks[i];
            if (b.kind != HLRC_LEAF_LOWRANK) continue;
            slabV[size_t(i)].push_back(st.alloc(b.V, b.ldv, tc.lo(t) - b.col0, tc.size(t), b.rank, cf(i), deffmt,
                                                nullptr, 1, wide16 ? int32_t(i) : -1));
        }
        st.close_region();
    }
    if (st.bytes >= (int64_t(1) << 36) && o.precision != HLRC_PREC_F64)
        return fail(HLRC_ERR_SHAPE, "reduced-precision store above 64 GiB");
    // FP64 plans hold FP64 chunks only, reduced-precision plans none: the two
    // kinds use different device descriptors
    for (const SChunk& ch : st.chunks)
        if ((ch.fmt == FMT_F64) != (o.precision == HLRC_PREC_F64))
            return fail(HLRC_ERR_INTERNAL, "chunk format %d in a plan of precision %d", ch.fmt, o.precision);
    if (o.leaves_on_device) {
        st.fill_device(p);
    } else {
        st.fill(p.store);
    }
    for (int f = 0; f < NFMT; ++f) p.fmt_bytes[f] = st.unpadded[f];

    p.npasses.resize(2);
    p.ttpasses.resize(3);
    // op N stage A: tile T-form V^T x -> t per column tile
    {
        TTPass& a = p.ttpasses[0];
        a.in = V_X; a.out = V_T; a.mode = OUT_SET;
        TTBuilder tb(a, st, size_t(nb));
        for (int64_t i = 0; i < nb; ++i)
            if (toff[size_t(i)] >= 0)
                tb.object(size_t(i), uint32_t(toff[size_t(i)]), d.blocks[i].rank,
                          tc.first(d.blocks[i].col0 + d.blocks[i].ncols) - tc.first(d.blocks[i].col0));
        for (int64_t t = 0; t < tc.n(); ++t) {
            tb.begin(tc.lo(t), tc.size(t));
            for (int64_t i : collist[size_t(t)]) {
                if (toff[size_t(i)] < 0) continue;
                const int64_t ti = t - tc.first(d.blocks[i].col0);
                tb.slab(slabV[size_t(i)][size_t(ti)], size_t(i), ti);
            }
            tb.end();
        }
        tb.finish();
    }
    // op N stage B: N-form per row tile, y += alpha (U t + D x)
    {
        NPass& nN = p.npasses[0];
        nN.vx = V_X; nN.vt = V_T; nN.out = V_Y; nN.mode = OUT_ADD_ALPHA;
        NBuilder nbld(nN, st);
        std::vector<size_t> pos(static_cast<size_t>(nb), 0);
        for (int64_t t = 0; t < tr.n(); ++t) {
            nbld.begin(tr.size(t));
            for (int64_t i : rowlist[size_t(t)]) {
                const hlrc_block& b = d.blocks[i];
                const int sid = slabA[size_t(i)][pos[size_t(i)]++];
                if (b.kind == HLRC_LEAF_DENSE) nbld.slab(sid, uint32_t(b.col0));
                else nbld.slab(sid, VEC_T | uint32_t(toff[size_t(i)]));
            }
            nbld.end(uint32_t(tr.lo(t)), tr.size(t), false);
        }
        nbld.finish();
    }
    // op T stage A: tile T-form U^T x -> t per row tile
    {
        TTPass& a = p.ttpasses[1];
        a.in = V_X; a.out = V_T; a.mode = OUT_SET;
        TTBuilder tb(a, st, size_t(nb));
        for (int64_t i = 0; i < nb; ++i)
            if (toff[size_t(i)] >= 0)
                tb.object(size_t(i), uint32_t(toff[size_t(i)]), d.blocks[i].rank,
                          tr.first(d.blocks[i].row0 + d.blocks[i].nrows) - tr.first(d.blocks[i].row0));
        for (int64_t t = 0; t < tr.n(); ++t) {
            tb.begin(tr.lo(t), tr.size(t));
            for (int64_t i : rowlist[size_t(t)]) {
                if (toff[size_t(i)] < 0) continue;
                const int64_t ti = t - tr.first(d.blocks[i].row0);
                tb.slab(slabA[size_t(i)][size_t(ti)], size_t(i), ti);
            }
            tb.end();
        }
        tb.finish();
    }
    // op T stage B: N-form per column tile, y += alpha V t
    {
        NPass& nT = p.npasses[1];
        nT.vx = V_X; nT.vt = V_T; nT.out = V_Y; nT.mode = OUT_ADD_ALPHA;
        NBuilder nbld(nT, st);
        for (int64_t t = 0; t < tc.n(); ++t) {
            nbld.begin(tc.size(t));
            for (int64_t i : collist[size_t(t)]) {
                const hlrc_block& b = d.blocks[i];
                if (b.kind != HLRC_LEAF_LOWRANK || toff[size_t(i)] < 0) continue;
                nbld.slab(slabV[size_t(i)][size_t(t - tc.first(b.col0))], VEC_T | uint32_t(toff[size_t(i)]));
            }
            nbld.end(uint32_t(tc.lo(t)), tc.size(t), false);
        }
        nbld.finish();
    }
    // op T near field: y += alpha D^T x
    plan_dense_transposed(p.ttpasses[2], st, tr, tc, dense_rows, slabA, [&](int64_t i, int64_t& c0, int64_t& nc) {
        c0 = d.blocks[i].col0;
        nc = d.blocks[i].ncols;
    });
    // op N with the near field on a side stream: y += alpha D x per row tile
    // (npasses[2]), then y += alpha U t (npasses[3]) after stage A
    if (g_knobs.side_dense(0)) {
        p.npasses.resize(4);
        for (int half = 0; half < 2; ++half) {
            NPass& q = p.npasses[size_t(2 + half)];
            q.vx = V_X; q.vt = V_T; q.out = V_Y; q.mode = OUT_ADD_ALPHA;
            NBuilder nbld(q, st);
            std::vector<size_t> pos(static_cast<size_t>(nb), 0);
            for (int64_t t = 0; t < tr.n(); ++t) {
                nbld.begin(tr.size(t));
                for (int64_t i : rowlist[size_t(t)]) {
                    const hlrc_block& b = d.blocks[i];
                    const int sid = slabA[size_t(i)][pos[size_t(i)]++];
                    const bool dense = b.kind == HLRC_LEAF_DENSE;
                    if (dense != (half == 0)) continue;
                    if (dense) nbld.slab(sid, uint32_t(b.col0));
                    else nbld.slab(sid, VEC_T | uint32_t(toff[size_t(i)]));
                }
                nbld.end(uint32_t(tr.lo(t)), tr.size(t), false);
            }
            nbld.finish();
        }
        p.stages_nf[HLRC_OP_N] = {{1, 2, 1}, {2, 0}, {1, 3}};
        p.nf_multi = g_knobs.near_field == 2;
    }
    p.stages[HLRC_OP_N] = {{2, 0}, {1, 0}};
    p.stages[HLRC_OP_T] = {{2, 1}, {1, 1}, {2, 2}};
    p.stages[HLRC_OP_C] = p.stages[HLRC_OP_T];
    for (const TTPass& tp : p.ttpasses)
        if (tp.npart >= (int64_t(1) << 32)) return fail(HLRC_ERR_SHAPE, "partial array exceeds 2^32 entries");
    if (wide16) {
        if (hlrc_status ws = plan_wide(d, tc, toff, cblk, slabV, st, p); ws != HLRC_OK) return ws;
    }

    if (hlrc_status vs = validate_plan(p); vs != HLRC_OK) return vs;

    // accounting (arith/mulvec.hh:795-874)
    double flops = 0;
    for (int64_t i = 0; i < nb; ++i) {
        const hlrc_block& b = d.blocks[i];
        if (b.kind == HLRC_LEAF_DENSE) {
            ++p.n_dense;
            flops += flops_gemv(double(b.nrows), double(b.ncols));
        } else {
            ++p.n_lowrank;
            flops += flops_gemv(double(b.ncols), b.rank) + flops_gemv(double(b.nrows), b.rank);
            p.max_rank = std::max(p.max_rank, b.rank);
        }
    }
    p.matrix_bytes = 0;
    for (int f = 0; f < NFMT; ++f) p.matrix_bytes += st.unpadded[f];
    p.algorithmic_bytes = p.matrix_bytes + 2 * 8 * (d.nrows + d.ncols);
    p.flops = int64_t(flops);
    return HLRC_OK;
}

// ------------------------------------------------------------- uniform-H
hlrc_status plan_uniform(const hlrc_uniform_desc& d, const hlrc_options& o, Plan& p) {
    if (hlrc_status ks = check_knobs(o); ks != HLRC_OK) return ks;
    if (o.leaves_on_device) return fail(HLRC_ERR_ARG, "leaves_on_device: H-matrix descriptors only");
    const KnobScope knobs(o);
    if (d.nrows < 0 || d.ncols < 0 || d.nblocks < 0 || d.nrow_bases < 0 || d.ncol_bases < 0)
        return fail(HLRC_ERR_SHAPE, "negative size");
    if ((d.nblocks > 0 && !d.blocks) || (d.nrow_bases > 0 && !d.row_bases) || (d.ncol_bases > 0 && !d.col_bases))
        return fail(HLRC_ERR_ARG, "NULL array in uniform descriptor");
    if (d.nrows >= (int64_t(1) << 31) || d.ncols >= (int64_t(1) << 31))
        return fail(HLRC_ERR_SHAPE, "matrix dimension exceeds 2^31-1");
    if (o.precision != HLRC_PREC_F64)
        return fail(HLRC_ERR_ARG, "precision %d not supported for uniform-H (FP64 only)", o.precision);
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

    std::vector<int64_t> rboff(static_cast<size_t>(nrb), -1), cboff(static_cast<size_t>(ncb), -1);
    int64_t nkr = 0, nkc = 0;
    for (int64_t i = 0; i < nrb; ++i)
        if (d.row_bases[i].rank > 0 && d.row_bases[i].size > 0) { rboff[size_t(i)] = nkr; nkr += d.row_bases[i].rank; }
    for (int64_t i = 0; i < ncb; ++i)
        if (d.col_bases[i].rank > 0 && d.col_bases[i].size > 0) { cboff[size_t(i)] = nkc; nkc += d.col_bases[i].rank; }
    if (std::max(nkr, nkc) >= (int64_t(1) << 31)) return fail(HLRC_ERR_SHAPE, "sum of basis ranks exceeds 2^31-1");
    p.n_t = std::max(nkr, nkc);
    p.n_t2 = std::max(nkr, nkc);

    // tile -> bases / dense blocks covering it
    std::vector<std::vector<int64_t>> rbl(static_cast<size_t>(tr.n())), cbl(static_cast<size_t>(tc.n())),
        rdl(static_cast<size_t>(tr.n()));
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
        } else {
            if (rboff[size_t(b.row_basis)] < 0 || cboff[size_t(b.col_basis)] < 0) continue;
            lr_by_row[size_t(b.row_basis)].push_back(i);
            lr_by_col[size_t(b.col_basis)].push_back(i);
        }
    }

    Store st;
    std::vector<std::vector<int>> sRB(static_cast<size_t>(nrb)), sCB(static_cast<size_t>(ncb)), sD(static_cast<size_t>(nb)),
        sS(static_cast<size_t>(nb));
    for (int64_t t = 0; t < tr.n(); ++t) {
        for (int64_t i : rbl[size_t(t)]) {
            const hlrc_basis& b = d.row_bases[i];
            sRB[size_t(i)].push_back(st.alloc(b.V, b.ldv, tr.lo(t) - b.ofs, tr.size(t), b.rank, nullptr, FMT_F64));
        }
        for (int64_t i : rdl[size_t(t)]) {
            const hlrc_uniform_block& b = d.blocks[i];
            const std::vector<int64_t> cuts = inner_cuts(tc, b.col0, b.ncols);
            sD[size_t(i)].push_back(st.alloc(b.D, b.ldd, tr.lo(t) - b.row0, tr.size(t), b.ncols, nullptr, FMT_F64, &cuts));
        }
    }
    for (int64_t t = 0; t < tc.n(); ++t)  // column bases by column tile
        for (int64_t i : cbl[size_t(t)]) {
            const hlrc_basis& b = d.col_bases[i];
            sCB[size_t(i)].push_back(st.alloc(b.V, b.ldv, tc.lo(t) - b.ofs, tc.size(t), b.rank, nullptr, FMT_F64));
        }
    for (int64_t i = 0; i < nb; ++i) {
        const hlrc_uniform_block& b = d.blocks[i];
        if (b.kind != HLRC_LEAF_LOWRANK || b.nrows == 0 || b.ncols == 0) continue;
        if (rboff[size_t(b.row_basis)] < 0 || cboff[size_t(b.col_basis)] < 0) continue;
        const int64_t kr = d.row_bases[b.row_basis].rank, kc = d.col_bases[b.col_basis].rank;
        for (int64_t r0 = 0; r0 < kr; r0 += TILE)
            sS[size_t(i)].push_back(st.alloc(b.S, b.lds, r0, std::min<int64_t>(TILE, kr - r0), kc, nullptr, FMT_F64));
    }
    st.close_region();   // one region: allocation order (FP64 only)
    st.fill(p.store);
    for (int f = 0; f < NFMT; ++f) p.fmt_bytes[f] = st.unpadded[f];

    p.tpasses.resize(1);
    p.npasses.resize(3);
    p.ttpasses.resize(3);
    // ---- op N
    {   // forward: ux_s = V_s^T x, per column tile over all bases containing it
        TTPass& f = p.ttpasses[0];
        f.in = V_X; f.out = V_T; f.mode = OUT_SET;
        TTBuilder tb(f, st, size_t(ncb));
        for (int64_t i = 0; i < ncb; ++i)
            if (cboff[size_t(i)] >= 0)
                tb.object(size_t(i), uint32_t(cboff[size_t(i)]), d.col_bases[i].rank,
                          tc.first(d.col_bases[i].ofs + d.col_bases[i].size) - tc.first(d.col_bases[i].ofs));
        for (int64_t t = 0; t < tc.n(); ++t) {
            tb.begin(tc.lo(t), tc.size(t));
            for (int64_t i : cbl[size_t(t)]) {
                const int64_t ti = t - tc.first(d.col_bases[i].ofs);
                tb.slab(sCB[size_t(i)][size_t(ti)], size_t(i), ti);
            }
            tb.end();
        }
        tb.finish();
    }
    {   // coupling: uy_t = sum_s S_ts ux_s
        NPass& c = p.npasses[0];
        c.vx = V_X; c.vt = V_T; c.out = V_T2; c.mode = OUT_SET;
        NBuilder nbld(c, st);
        for (int64_t t = 0; t < nrb; ++t) {
            if (rboff[size_t(t)] < 0) continue;
            const int64_t kr = d.row_bases[t].rank;
            for (int64_t r0 = 0, piece = 0; r0 < kr; r0 += TILE, ++piece) {
                const int64_t rows = std::min<int64_t>(TILE, kr - r0);
                nbld.begin(rows);
                for (int64_t i : lr_by_row[size_t(t)]) {
                    const hlrc_uniform_block& b = d.blocks[i];
                    nbld.slab(sS[size_t(i)][size_t(piece)], VEC_T | uint32_t(cboff[size_t(b.col_basis)]));
                }
                nbld.end(uint32_t(rboff[size_t(t)] + r0), rows, true);
            }
        }
        nbld.finish();
    }
    {   // backward + near field: y_tau += alpha (sum_t V_t[tau] uy_t + sum D x)
        NPass& bw = p.npasses[1];
        bw.vx = V_X; bw.vt = V_T2; bw.out = V_Y; bw.mode = OUT_ADD_ALPHA;
        NBuilder nbld(bw, st);
        std::vector<size_t> posRB(static_cast<size_t>(nrb), 0), posD(static_cast<size_t>(nb), 0);
        for (int64_t t = 0; t < tr.n(); ++t) {
            nbld.begin(tr.size(t));
            for (int64_t i : rbl[size_t(t)]) nbld.slab(sRB[size_t(i)][posRB[size_t(i)]++], VEC_T | uint32_t(rboff[size_t(i)]));
            for (int64_t i : rdl[size_t(t)]) nbld.slab(sD[size_t(i)][posD[size_t(i)]++], uint32_t(d.blocks[i].col0));
            nbld.end(uint32_t(tr.lo(t)), tr.size(t), false);
        }
        nbld.finish();
    }
    // ---- op C (adjoint)
    {   // forward with row bases: ux'_t = V_t^T x, per row tile
        TTPass& f = p.ttpasses[1];
        f.in = V_X; f.out = V_T; f.mode = OUT_SET;
        TTBuilder tb(f, st, size_t(nrb));
        for (int64_t i = 0; i < nrb; ++i)
            if (rboff[size_t(i)] >= 0)
                tb.object(size_t(i), uint32_t(rboff[size_t(i)]), d.row_bases[i].rank,
                          tr.first(d.row_bases[i].ofs + d.row_bases[i].size) - tr.first(d.row_bases[i].ofs));
        for (int64_t t = 0; t < tr.n(); ++t) {
            tb.begin(tr.lo(t), tr.size(t));
            for (int64_t i : rbl[size_t(t)]) {
                const int64_t ti = t - tr.first(d.row_bases[i].ofs);
                tb.slab(sRB[size_t(i)][size_t(ti)], size_t(i), ti);
            }
            tb.end();
        }
        tb.finish();
    }
    {   // coupling^T: uy'_s = sum_t S_ts^T ux'_t (coefficient vectors are small: unit T-form)
        TPass& c = p.tpasses[0];
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
                    sl.push_back({uint64_t(st.slab_elem_off(sS[size_t(i)][size_t(piece)])),
                                  uint32_t(rboff[size_t(b.row_basis)] + r0), uint16_t(rows), uint16_t(pad_rows(rows))});
                }
            }
            tb.add(uint32_t(cboff[size_t(s)]), d.col_bases[s].rank, sl);
        }
        tb.finish();
    }
    {   // backward with column bases: y_sigma += alpha sum_s V_s[sigma] uy'_s
        NPass& bw = p.npasses[2];
        bw.vx = V_X; bw.vt = V_T2; bw.out = V_Y; bw.mode = OUT_ADD_ALPHA;
        NBuilder nbld(bw, st);
        for (int64_t t = 0; t < tc.n(); ++t) {
            nbld.begin(tc.size(t));
            for (int64_t i : cbl[size_t(t)])
                nbld.slab(sCB[size_t(i)][size_t(t - tc.first(d.col_bases[i].ofs))], VEC_T | uint32_t(cboff[size_t(i)]));
            nbld.end(uint32_t(tc.lo(t)), tc.size(t), false);
        }
        nbld.finish();
    }
    // near field transposed: y_sigma += alpha sum D^T x
    plan_dense_transposed(p.ttpasses[2], st, tr, tc, rdl, sD, [&](int64_t i, int64_t& c0, int64_t& nc) {
        c0 = d.blocks[i].col0;
        nc = d.blocks[i].ncols;
    });
    // op N with the near field on a side stream: y += alpha D x per row tile
    // (npasses[3]), then y += alpha V_t uy_t (npasses[4]) after the coupling
    if (g_knobs.side_dense(1)) {
        p.npasses.resize(5);
        for (int half = 0; half < 2; ++half) {
            NPass& q = p.npasses[size_t(3 + half)];
            q.vx = V_X; q.vt = V_T2; q.out = V_Y; q.mode = OUT_ADD_ALPHA;
            NBuilder nbld(q, st);
            std::vector<size_t> posRB(static_cast<size_t>(nrb), 0), posD(static_cast<size_t>(nb), 0);
            for (int64_t t = 0; t < tr.n(); ++t) {
                nbld.begin(tr.size(t));
                if (half == 1)
                    for (int64_t i : rbl[size_t(t)])
                        nbld.slab(sRB[size_t(i)][posRB[size_t(i)]++], VEC_T | uint32_t(rboff[size_t(i)]));
                if (half == 0)
                    for (int64_t i : rdl[size_t(t)]) nbld.slab(sD[size_t(i)][posD[size_t(i)]++], uint32_t(d.blocks[i].col0));
                nbld.end(uint32_t(tr.lo(t)), tr.size(t), false);
            }
            nbld.finish();
        }
        p.stages_nf[HLRC_OP_N] = {{1, 3, 1}, {2, 0}, {1, 0}, {1, 4}};
        p.nf_multi = g_knobs.near_field == 2;
    }
    p.stages[HLRC_OP_N] = {{2, 0}, {1, 0}, {1, 1}};
    p.stages[HLRC_OP_T].clear();  // uniform_lrmatrix::uni_apply_add asserts on apply_transposed
    p.stages[HLRC_OP_C] = {{2, 1}, {0, 0}, {1, 2}, {2, 2}};
    for (const TTPass& tp : p.ttpasses)
        if (tp.npart >= (int64_t(1) << 32)) return fail(HLRC_ERR_SHAPE, "partial array exceeds 2^32 entries");

    if (hlrc_status vs = validate_plan(p); vs != HLRC_OK) return vs;

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

// ------------------------------------------------------------------- H^2
// The product of an H^2 matrix as a sequence of the same N-form and tile
// T-form passes (arith/h2.hh:21-40, arith/detail/h2.hh:238-330).  op N:
//   1. x^_s = W_s^T x for the leaf column clusters             (tile T-form)
//   2. per level of the column tree, deepest first:
//      x^_p = sum over the sons s of F_s^T x^_s                 (N-form over
//      the transposed transfer matrices, one output per parent)
//   3. y^_t = sum_s S_ts x^_s for every row cluster (zero if none)  (N-form)
//   4. per level of the row tree, root first:
//      y^_c += E_c y^_p for the sons c of the level's clusters  (N-form, add)
//   5. y += alpha (V_t y^_t over the leaf row clusters + D x)    (N-form)
// op C exchanges the trees: forward with the row bases, the couplings
// transposed (unit T-form), backward down the column tree, leaf column
// bases, and the near field transposed.
hlrc_status plan_h2(const hlrc_h2_desc& d, const hlrc_options& o, Plan& p) {
    if (hlrc_status ks = check_knobs(o); ks != HLRC_OK) return ks;
    if (o.leaves_on_device) return fail(HLRC_ERR_ARG, "leaves_on_device: H-matrix descriptors only");
    const KnobScope knobs(o);
    if (d.nrows < 0 || d.ncols < 0 || d.nblocks < 0 || d.nrow_clusters <= 0 || d.ncol_clusters <= 0)
        return fail(HLRC_ERR_SHAPE, "H2: bad sizes or empty cluster tree");
    if ((d.nblocks > 0 && !d.blocks) || !d.row_clusters || !d.col_clusters)
        return fail(HLRC_ERR_ARG, "H2: NULL array in descriptor");
    if (d.nrows >= (int64_t(1) << 31) || d.ncols >= (int64_t(1) << 31))
        return fail(HLRC_ERR_SHAPE, "matrix dimension exceeds 2^31-1");
    if (o.precision != HLRC_PREC_F64)
        return fail(HLRC_ERR_ARG, "precision %d not supported for H2 (FP64 only)", o.precision);
    p = Plan();
    p.kind = 2;
    p.precision = o.precision;
    p.nrows = d.nrows;
    p.ncols = d.ncols;
    const int64_t nb = d.nblocks;
    // ---- cluster trees: index sets, parent/son links, levels, data
    struct Tree {
        const hlrc_h2_cluster* c;
        int64_t n;
        std::vector<int> level;
        std::vector<int64_t> off;   // coefficient offsets (-1: rank 0)
        int64_t ncoef = 0;
        int maxlev = 0;
        bool leaf(int64_t t) const { return c[t].son[0] < 0 && c[t].son[1] < 0; }
    };
    auto check_tree = [&](const hlrc_h2_cluster* cl, int64_t n, int64_t dim, Tree& T, const char* side) -> hlrc_status {
        T.c = cl; T.n = n;
        T.level.assign(size_t(n), -1);
        T.off.assign(size_t(n), -1);
        if (cl[0].parent != -1 || cl[0].ofs != 0 || cl[0].size != dim)
            return fail(HLRC_ERR_SHAPE, "H2 %s tree: cluster 0 must be the root covering all indices", side);
        std::vector<int64_t> stack{0};
        T.level[0] = 0;
        int64_t seen = 0;
        while (!stack.empty()) {
            const int64_t t = stack.back();
            stack.pop_back();
            ++seen;
            const hlrc_h2_cluster& c = cl[t];
            if (c.ofs < 0 || c.size < 0 || c.ofs + c.size > dim || c.rank < 0 || c.rank > 65535)
                return fail(HLRC_ERR_SHAPE, "H2 %s cluster %lld: bad index set or rank", side, (long long)t);
            const bool lf = c.son[0] < 0 && c.son[1] < 0;
            if (lf && c.rank > 0 && c.size > 0 && (!c.V || c.ldv < c.size))
                return fail(HLRC_ERR_ARG, "H2 %s cluster %lld: leaf basis missing", side, (long long)t);
            if (t != 0) {
                const int64_t pr = c.parent;
                if (c.rank > 0 && cl[pr].rank > 0 && (!c.E || c.lde < c.rank))
                    return fail(HLRC_ERR_ARG, "H2 %s cluster %lld: transfer matrix missing", side, (long long)t);
            }
            int64_t covered = 0;
            for (int i = 0; i < 2; ++i) {
                const int64_t s = c.son[i];
                if (s < 0) continue;
                if (s >= n || cl[s].parent != t || T.level[size_t(s)] >= 0)
                    return fail(HLRC_ERR_SHAPE, "H2 %s cluster %lld: inconsistent son %lld", side, (long long)t, (long long)s);
                if (cl[s].ofs != c.ofs + covered)
                    return fail(HLRC_ERR_SHAPE, "H2 %s cluster %lld: sons do not partition it", side, (long long)t);
                covered += cl[s].size;
                T.level[size_t(s)] = T.level[size_t(t)] + 1;
                T.maxlev = std::max(T.maxlev, T.level[size_t(s)]);
                stack.push_back(s);
            }
            if (!lf && covered != c.size)
                return fail(HLRC_ERR_SHAPE, "H2 %s cluster %lld: sons do not partition it", side, (long long)t);
            if (!lf && c.rank > 0 && !((c.son[0] >= 0 && cl[c.son[0]].rank > 0) || (c.son[1] >= 0 && cl[c.son[1]].rank > 0)))
                return fail(HLRC_ERR_SHAPE, "H2 %s cluster %lld: positive rank but no son of positive rank", side,
                            (long long)t);
        }
        if (seen != n) return fail(HLRC_ERR_SHAPE, "H2 %s tree: %lld clusters unreachable from the root", side,
                                    (long long)(n - seen));
        for (int64_t t = 0; t < n; ++t)
            if (cl[t].rank > 0) { T.off[size_t(t)] = T.ncoef; T.ncoef += cl[t].rank; }
        return HLRC_OK;
    };
    Tree R, Cc;
    if (hlrc_status st = check_tree(d.row_clusters, d.nrow_clusters, d.nrows, R, "row"); st != HLRC_OK) return st;
    if (hlrc_status st = check_tree(d.col_clusters, d.ncol_clusters, d.ncols, Cc, "column"); st != HLRC_OK) return st;
    if (std::max(R.ncoef, Cc.ncoef) >= (int64_t(1) << 31)) return fail(HLRC_ERR_SHAPE, "sum of basis ranks exceeds 2^31-1");
    // ---- blocks
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
            if (b.row_basis < 0 || b.row_basis >= R.n || b.col_basis < 0 || b.col_basis >= Cc.n)
                return fail(HLRC_ERR_ARG, "block %lld: cluster index out of range", (long long)i);
            const hlrc_h2_cluster& rc = R.c[b.row_basis];
            const hlrc_h2_cluster& cc = Cc.c[b.col_basis];
            if (rc.ofs != b.row0 || rc.size != b.nrows || cc.ofs != b.col0 || cc.size != b.ncols)
                return fail(HLRC_ERR_SHAPE, "block %lld: cluster index sets differ from the block's", (long long)i);
            if (rc.rank > 0 && cc.rank > 0 && (!b.S || b.lds < rc.rank))
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
    for (int64_t t = 0; t < R.n; ++t)
        if (R.leaf(t)) { rcuts.push_back(R.c[t].ofs); rcuts.push_back(R.c[t].ofs + R.c[t].size); }
    for (int64_t t = 0; t < Cc.n; ++t)
        if (Cc.leaf(t)) { ccuts.push_back(Cc.c[t].ofs); ccuts.push_back(Cc.c[t].ofs + Cc.c[t].size); }
    const Tiles tr = make_tiles(d.nrows, rcuts), tc = make_tiles(d.ncols, ccuts);
    p.n_row_tiles = tr.n();
    p.n_col_tiles = tc.n();
    p.n_t = p.n_t2 = std::max(R.ncoef, Cc.ncoef);

    // tiles -> leaf bases / dense blocks; clusters -> low-rank blocks
    std::vector<std::vector<int64_t>> rbl(static_cast<size_t>(tr.n())), cbl(static_cast<size_t>(tc.n())),
        rdl(static_cast<size_t>(tr.n()));
    for (int64_t t = 0; t < R.n; ++t)
        if (R.leaf(t) && R.c[t].rank > 0)
            for (int64_t q = tr.first(R.c[t].ofs); q < tr.first(R.c[t].ofs + R.c[t].size); ++q) rbl[size_t(q)].push_back(t);
    for (int64_t t = 0; t < Cc.n; ++t)
        if (Cc.leaf(t) && Cc.c[t].rank > 0)
            for (int64_t q = tc.first(Cc.c[t].ofs); q < tc.first(Cc.c[t].ofs + Cc.c[t].size); ++q) cbl[size_t(q)].push_back(t);
    std::vector<std::vector<int64_t>> lr_by_row(static_cast<size_t>(R.n)), lr_by_col(static_cast<size_t>(Cc.n));
    for (int64_t i = 0; i < nb; ++i) {
        const hlrc_uniform_block& b = d.blocks[i];
        if (b.nrows == 0 || b.ncols == 0) continue;
        if (b.kind == HLRC_LEAF_DENSE) {
            for (int64_t q = tr.first(b.row0); q < tr.first(b.row0 + b.nrows); ++q) rdl[size_t(q)].push_back(i);
        } else if (R.c[b.row_basis].rank > 0 && Cc.c[b.col_basis].rank > 0) {
            lr_by_row[size_t(b.row_basis)].push_back(i);
            lr_by_col[size_t(b.col_basis)].push_back(i);
        }
    }

    // ---- storage (FP64): leaf bases by tile, dense slabs, couplings and
    // transfer matrices in pieces of at most TILE rows
    Store st;
    std::vector<std::vector<int>> sRB(static_cast<size_t>(R.n)), sCB(static_cast<size_t>(Cc.n)),
        sER(static_cast<size_t>(R.n)), sEC(static_cast<size_t>(Cc.n)), sD(static_cast<size_t>(nb)),
        sS(static_cast<size_t>(nb));
    for (int64_t q = 0; q < tr.n(); ++q) {
        for (int64_t t : rbl[size_t(q)]) {
            const hlrc_h2_cluster& c = R.c[t];
            sRB[size_t(t)].push_back(st.alloc(c.V, c.ldv, tr.lo(q) - c.ofs, tr.size(q), c.rank, nullptr, FMT_F64));
        }
        for (int64_t i : rdl[size_t(q)]) {
            const hlrc_uniform_block& b = d.blocks[i];
            const std::vector<int64_t> cuts = inner_cuts(tc, b.col0, b.ncols);
            sD[size_t(i)].push_back(st.alloc(b.D, b.ldd, tr.lo(q) - b.row0, tr.size(q), b.ncols, nullptr, FMT_F64, &cuts));
        }
    }
    for (int64_t q = 0; q < tc.n(); ++q)
        for (int64_t t : cbl[size_t(q)]) {
            const hlrc_h2_cluster& c = Cc.c[t];
            sCB[size_t(t)].push_back(st.alloc(c.V, c.ldv, tc.lo(q) - c.ofs, tc.size(q), c.rank, nullptr, FMT_F64));
        }
    auto pieces = [&](const double* A, int64_t lda, int64_t rows, int64_t cols, std::vector<int>& out) {
        for (int64_t r0 = 0; r0 < rows; r0 += TILE)
            out.push_back(st.alloc(A, lda, r0, std::min<int64_t>(TILE, rows - r0), cols, nullptr, FMT_F64));
    };
    for (int64_t i = 0; i < nb; ++i) {
        const hlrc_uniform_block& b = d.blocks[i];
        if (b.kind != HLRC_LEAF_LOWRANK || b.nrows == 0 || b.ncols == 0) continue;
        const int64_t kr = R.c[b.row_basis].rank, kc = Cc.c[b.col_basis].rank;
        if (kr > 0 && kc > 0) pieces(b.S, b.lds, kr, kc, sS[size_t(i)]);
    }
    auto transfer_ok = [](const Tree& T, int64_t t) {
        return t != 0 && T.c[t].rank > 0 && T.c[T.c[t].parent].rank > 0;
    };
    for (int64_t t = 0; t < R.n; ++t)
        if (transfer_ok(R, t)) pieces(R.c[t].E, R.c[t].lde, R.c[t].rank, R.c[R.c[t].parent].rank, sER[size_t(t)]);
    for (int64_t t = 0; t < Cc.n; ++t)
        if (transfer_ok(Cc, t)) pieces(Cc.c[t].E, Cc.c[t].lde, Cc.c[t].rank, Cc.c[Cc.c[t].parent].rank, sEC[size_t(t)]);
    // the forward transform takes the transposed transfer matrices (parent
    // rank x son rank), so that a parent's coefficients are one N-form
    // output over both sons, with no partial sums
    std::vector<std::vector<double>> ET(static_cast<size_t>(R.n + Cc.n));
    std::vector<std::vector<int>> sETR(static_cast<size_t>(R.n)), sETC(static_cast<size_t>(Cc.n));
    auto transposed = [&](const hlrc_h2_cluster& c, int64_t kp, std::vector<double>& buf) {
        buf.assign(size_t(kp * c.rank), 0.0);
        for (int64_t j = 0; j < kp; ++j)
            for (int64_t i = 0; i < c.rank; ++i) buf[size_t(j + i * kp)] = c.E[i + j * c.lde];
    };
    for (int64_t t = 0; t < R.n; ++t)
        if (transfer_ok(R, t)) {
            const int64_t kp = R.c[R.c[t].parent].rank;
            transposed(R.c[t], kp, ET[size_t(t)]);
            pieces(ET[size_t(t)].data(), kp, kp, R.c[t].rank, sETR[size_t(t)]);
        }
    for (int64_t t = 0; t < Cc.n; ++t)
        if (transfer_ok(Cc, t)) {
            const int64_t kp = Cc.c[Cc.c[t].parent].rank;
            transposed(Cc.c[t], kp, ET[size_t(R.n + t)]);
            pieces(ET[size_t(R.n + t)].data(), kp, kp, Cc.c[t].rank, sETC[size_t(t)]);
        }
    st.close_region();   // one region: allocation order (FP64 only)
    st.fill(p.store);
    for (int f = 0; f < NFMT; ++f) p.fmt_bytes[f] = st.unpadded[f];

    // ---- pass builders
    // forward leaf transform of a tree over its tiles: x^_s = W_s^T x
    auto fwd_leaves = [&](TTPass& f, const Tree& T, const Tiles& tl, const std::vector<std::vector<int64_t>>& bl,
                          const std::vector<std::vector<int>>& sB) {
        f.in = V_X; f.out = V_T; f.mode = OUT_SET;
        TTBuilder tb(f, st, size_t(T.n));
        for (int64_t t = 0; t < T.n; ++t)
            if (T.leaf(t) && T.c[t].rank > 0)
                tb.object(size_t(t), uint32_t(T.off[size_t(t)]), T.c[t].rank,
                          tl.first(T.c[t].ofs + T.c[t].size) - tl.first(T.c[t].ofs));
        for (int64_t q = 0; q < tl.n(); ++q) {
            tb.begin(tl.lo(q), tl.size(q));
            for (int64_t t : bl[size_t(q)]) tb.slab(sB[size_t(t)][size_t(q - tl.first(T.c[t].ofs))], size_t(t), q - tl.first(T.c[t].ofs));
            tb.end();
        }
        tb.finish();
    };
    // forward transfer into parent t: x^_t = sum_s E_s^T x^_s, one N-form
    // output (pieces of at most TILE rows) over the transposed transfer
    // matrices of its sons
    auto fwd_parent = [&](NBuilder& nbld, const Tree& T, const std::vector<std::vector<int>>& sET, int64_t t) -> bool {
        if (T.leaf(t) || T.c[t].rank == 0) return false;
        const int64_t kp = T.c[t].rank;
        for (int64_t r0 = 0, piece = 0; r0 < kp; r0 += TILE, ++piece) {
            const int64_t rows = std::min<int64_t>(TILE, kp - r0);
            nbld.begin(rows);
            for (int i = 0; i < 2; ++i) {
                const int64_t so = T.c[t].son[i];
                if (so >= 0 && !sET[size_t(so)].empty())
                    nbld.slab(sET[size_t(so)][size_t(piece)], VEC_T | uint32_t(T.off[size_t(so)]));
            }
            nbld.end(uint32_t(T.off[size_t(t)] + r0), rows, true);
        }
        return true;
    };
    // backward transfer into son c: y^_c += E_c y^_p
    auto bwd_child = [&](NBuilder& nbld, const Tree& T, const std::vector<std::vector<int>>& sE, int64_t c) -> bool {
        if (sE[size_t(c)].empty()) return false;
        const int64_t pr = T.c[c].parent;
        for (size_t pc = 0; pc < sE[size_t(c)].size(); ++pc) {
            const int64_t r0 = int64_t(pc) * TILE, rows = std::min<int64_t>(TILE, T.c[c].rank - r0);
            nbld.begin(rows);
            nbld.slab(sE[size_t(c)][pc], VEC_T | uint32_t(T.off[size_t(pr)]));
            nbld.end(uint32_t(T.off[size_t(c)] + r0), rows, false);
        }
        return true;
    };
    // one pass per level: the forward transfers into the clusters of level
    // lev, the backward transfers into the sons of level lev
    auto fwd_transfer = [&](NPass& n, const Tree& T, const std::vector<std::vector<int>>& sET, int lev) -> bool {
        n.vx = V_X; n.vt = V_T; n.out = V_T; n.mode = OUT_SET;
        NBuilder nbld(n, st);
        bool any = false;
        for (int64_t t = 0; t < T.n; ++t)
            if (T.level[size_t(t)] == lev) any |= fwd_parent(nbld, T, sET, t);
        nbld.finish();
        return any;
    };
    auto bwd_transfer = [&](NPass& n, const Tree& T, const std::vector<std::vector<int>>& sE, int lev) -> bool {
        n.vx = V_X; n.vt = V_T2; n.out = V_T2; n.mode = OUT_ADD;
        NBuilder nbld(n, st);
        bool any = false;
        for (int64_t c = 0; c < T.n; ++c)
            if (T.level[size_t(c)] == lev + 1) any |= bwd_child(nbld, T, sE, c);
        nbld.finish();
        return any;
    };
    // tree sweep: the levels lo..hi of every subtree rooted at level L0 in
    // one pass, one CTA cluster per subtree, deepest level first (up) or
    // shallowest first; emit adds a cluster's segments.  Fails when a
    // subtree does not fit the CTAs' shared memory.
    auto tree_pass = [&](NPass& n, const Tree& T, int L0, int lo, int hi, bool up, auto&& emit) -> bool {
        NBuilder nbld(n, st);
        nbld.keep_order = true;
        n.cta_begin.assign(1, 0);
        n.tree_level.assign(1, 0);
        for (int64_t r = 0; r < T.n; ++r) {
            if (T.level[size_t(r)] != L0) continue;
            std::vector<std::vector<int64_t>> lv(size_t(T.maxlev) + 1);
            for (std::vector<int64_t> stack{r}; !stack.empty();) {
                const int64_t t = stack.back();
                stack.pop_back();
                lv[size_t(T.level[size_t(t)])].push_back(t);
                for (int i = 0; i < 2; ++i)
                    if (T.c[t].son[i] >= 0) stack.push_back(T.c[t].son[i]);
            }
            for (int k = 0; k <= hi - lo; ++k) {
                std::vector<int64_t>& v = lv[size_t(up ? hi - k : lo + k)];
                std::sort(v.begin(), v.end());
                for (int64_t t : v) emit(nbld, t);
                const int32_t ns = int32_t(nbld.tmp[FMT_F64].size());
                if (ns > n.tree_level.back()) n.tree_level.push_back(ns);
            }
            const int32_t nl = int32_t(n.tree_level.size()) - 1;
            if (nl > n.cta_begin.back()) n.cta_begin.push_back(nl);
        }
        nbld.finish();
        if (n.cta_begin.size() < 2) return false;
        // per subtree: each level's segments split into TREE_CLUSTER runs of
        // about equal bytes (one per cluster rank); stage offsets of the
        // chunks in their owner's stage; mirror slots for the rows of the
        // segments, then for the coefficients read from outside (the leaves'
        // or the subtree root's), one run per chunk
        const std::vector<NSeg>& sg = n.segs[FMT_F64];
        const std::vector<int32_t>& tl = n.tree_level;
        constexpr int TC = TREE_CLUSTER;
        auto seg_bytes = [&](int32_t q) { return int64_t(sg[size_t(q)].ce - sg[size_t(q)].cb) * sg[size_t(q)].ld; };
        n.tree_part.assign((tl.size() - 1) * (TC + 1), 0);
        n.tree_seg.assign(sg.size(), 0);
        n.tree_chunk.assign(n.chunks.size(), TreeChunk{0, 0});
        n.tree_ext.clear();
        n.tree_cta_ext.assign(1, 0);
        n.tree_stage = n.tree_mirror = 0;
        n.tree_levels = n.tree_segs = n.tree_chunks = n.tree_items = 0;
        for (size_t b = 0; b + 1 < n.cta_begin.size(); ++b) {
            const int32_t s0 = tl[size_t(n.cta_begin[b])], s1 = tl[size_t(n.cta_begin[b + 1])];
            uint32_t rows = 0;
            for (int32_t q = s0; q < s1; ++q) {
                n.tree_seg[size_t(q)] = int32_t(rows);
                rows += sg[size_t(q)].rows;
            }
            uint32_t next = rows;
            uint32_t stage[TC] = {};
            int64_t load[TC] = {};   // stage doubles per rank so far
            std::unordered_map<uint32_t, uint32_t> made;   // coefficient -> mirror slot, earlier levels
            for (int32_t g = n.cta_begin[b]; g < n.cta_begin[b + 1]; ++g) {
                const int32_t q0 = tl[size_t(g)], q1 = tl[size_t(g) + 1];
                int64_t tot = 0;
                for (int32_t q = q0; q < q1; ++q) tot += seg_bytes(q);
                int32_t* part = &n.tree_part[size_t(g) * (TC + 1)];
                part[0] = q0;
                if (q1 - q0 <= TC) {   // one segment each for the least loaded ranks, in rank order
                    int rk[TC];
                    std::iota(rk, rk + TC, 0);
                    std::stable_sort(rk, rk + TC, [&](int x, int y) { return load[x] < load[y]; });
                    std::sort(rk, rk + (q1 - q0));
                    int32_t q = q0;
                    for (int r = 0, k = 0; r < TC; ++r) {
                        if (k < q1 - q0 && rk[k] == r) { load[r] += seg_bytes(q++); ++k; }
                        part[r + 1] = q;
                    }
                } else {   // runs of about equal bytes, rank r until its share is reached
                    int64_t acc = 0;
                    int32_t q = q0;
                    for (int r = 0; r < TC; ++r) {
                        const int64_t a0 = acc;
                        while (q < q1 && (r == TC - 1 || acc * TC < tot * (r + 1) || acc == 0)) acc += seg_bytes(q++);
                        part[r + 1] = q;
                        load[r] += acc - a0;
                    }
                }
                for (int r = 0; r < TC; ++r) {
                    int items = 0;
                    for (int32_t qq = part[r]; qq < part[r + 1]; ++qq)
                        for (uint32_t c = sg[size_t(qq)].cb; c < sg[size_t(qq)].ce; ++c) {
                            const GChunk& ch = n.chunks[c];
                            TreeChunk& tc = n.tree_chunk[c];
                            tc.stage = stage[r];
                            stage[r] += uint32_t(ch.nc) * sg[size_t(qq)].ld;
                            ++items;
                            const auto f0 = made.find(ch.vo);
                            bool run = f0 != made.end();
                            for (uint32_t j = 1; j < ch.nc && run; ++j) {
                                const auto fj = made.find(ch.vo + j);
                                run = fj != made.end() && fj->second == f0->second + j;
                            }
                            if (run) {
                                tc.mirror = f0->second;
                            } else {
                                tc.mirror = next;
                                for (uint32_t j = 0; j < ch.nc; ++j) n.tree_ext.push_back(TreeExt{next++, ch.vo + j});
                            }
                        }
                    n.tree_items = std::max(n.tree_items, items);
                }
                for (int32_t qq = q0; qq < q1; ++qq)
                    for (uint32_t i = 0; i < sg[size_t(qq)].rows; ++i)
                        made[(VEC_T | sg[size_t(qq)].out) + i] = uint32_t(n.tree_seg[size_t(qq)]) + i;
            }
            n.tree_cta_ext.push_back(int32_t(n.tree_ext.size()));
            for (int r = 0; r < TC; ++r) n.tree_stage = std::max<int64_t>(n.tree_stage, stage[r]);
            n.tree_mirror = std::max<int64_t>(n.tree_mirror, next);
            n.tree_levels = std::max(n.tree_levels, int(n.cta_begin[b + 1] - n.cta_begin[b]));
            n.tree_segs = std::max(n.tree_segs, int(s1 - s0));
            n.tree_chunks = std::max(n.tree_chunks, int(sg[size_t(s1 - 1)].ce - sg[size_t(s0)].cb));
        }
        return tree_smem_bytes(n.tree_stage, n.tree_mirror, n.tree_levels, n.tree_segs, n.tree_chunks,
                               n.tree_items) <= TREE_SMEM;
    };
    // subtrees rooted at the first level with at least TREE_MIN_SUBTREES
    // clusters, or deeper while a level of a subtree holds too many chunks;
    // -1 when fewer than two levels would be swept
    auto tree_root = [&](const Tree& T) -> int {
        std::vector<int64_t> cnt(size_t(T.maxlev) + 1, 0);
        for (int64_t t = 0; t < T.n; ++t) ++cnt[size_t(T.level[size_t(t)])];
        for (int l = 0; l <= T.maxlev; ++l)
            if (cnt[size_t(l)] >= TREE_MIN_SUBTREES) return l;
        return -1;
    };
    // backward leaf transform (+ near field for op N): y += alpha (V_t y^_t + D x)
    auto bwd_leaves = [&](NPass& n, const Tree& T, const Tiles& tl, const std::vector<std::vector<int64_t>>& bl,
                          const std::vector<std::vector<int>>& sB, bool dense) {
        n.vx = V_X; n.vt = V_T2; n.out = V_Y; n.mode = OUT_ADD_ALPHA;
        NBuilder nbld(n, st);
        std::vector<size_t> posD(static_cast<size_t>(nb), 0);
        for (int64_t q = 0; q < tl.n(); ++q) {
            nbld.begin(tl.size(q));
            for (int64_t t : bl[size_t(q)])
                nbld.slab(sB[size_t(t)][size_t(q - tl.first(T.c[t].ofs))], VEC_T | uint32_t(T.off[size_t(t)]));
            if (dense)
                for (int64_t i : rdl[size_t(q)]) nbld.slab(sD[size_t(i)][posD[size_t(i)]++], uint32_t(d.blocks[i].col0));
            nbld.end(uint32_t(tl.lo(q)), tl.size(q), false);
        }
        nbld.finish();
    };

    auto add_tt = [&](const char* name) -> TTPass& {
        p.ttpasses.emplace_back();
        p.names[2].push_back(name);
        return p.ttpasses.back();
    };
    auto add_n = [&](const char* name) -> NPass& {
        p.npasses.emplace_back();
        p.names[1].push_back(name);
        return p.npasses.back();
    };
    auto drop_n = [&]() { p.npasses.pop_back(); p.names[1].pop_back(); };
    // passes are appended, so stages record indices, not references.  Every
    // level has its own pass (the multi-vector product runs those); the
    // one-vector product runs the levels of the subtrees in one tree sweep
    // per tree when one can be built.
    // up: forward leaves + transfers of tree Tf; down: backward transfers of
    // tree Tb.  `mid` is the coupling stage between them.
    auto compose = [&](int op, const Tree& Tf, const std::vector<std::vector<int>>& sETf, const Tree& Tb,
                       const std::vector<std::vector<int>>& sEb, const Stage& leaves_in, const Stage& mid,
                       const std::vector<Stage>& tail) {
        std::vector<int> up(size_t(Tf.maxlev) + 1, -1), down(size_t(Tb.maxlev) + 1, -1);
        for (int lev = Tf.maxlev - 1; lev >= 0; --lev) {
            if (fwd_transfer(add_n("h2_fwd_transfer"), Tf, sETf, lev)) up[size_t(lev)] = int(p.npasses.size()) - 1;
            else drop_n();
        }
        for (int lev = 0; lev < Tb.maxlev; ++lev) {
            if (bwd_transfer(add_n("h2_bwd_transfer"), Tb, sEb, lev)) down[size_t(lev)] = int(p.npasses.size()) - 1;
            else drop_n();
        }
        // forward sweep: parents at levels L0..maxlev-1 of the subtrees
        int upL0 = -1, upIdx = -1, downL0 = -1, downIdx = -1;
        for (int L0 = tree_root(Tf); L0 >= 0 && L0 + 1 <= Tf.maxlev - 1 && upIdx < 0; ++L0) {
            NPass& n = add_n("h2_fwd_tree");
            n.vx = V_X; n.vt = V_T; n.out = V_T; n.mode = OUT_SET;
            if (tree_pass(n, Tf, L0, L0, Tf.maxlev - 1, true,
                          [&](NBuilder& nb, int64_t t) { fwd_parent(nb, Tf, sETf, t); })) {
                upL0 = L0;
                upIdx = int(p.npasses.size()) - 1;
            } else {
                drop_n();
            }
        }
        // backward sweep: sons at levels L0..maxlev of the subtrees; a
        // subtree root's own transfer reads its parent's y^, which the
        // passes before the sweep complete
        for (int L0 = tree_root(Tb); L0 >= 0 && L0 + 2 <= Tb.maxlev && downIdx < 0; ++L0) {
            NPass& n = add_n("h2_bwd_tree");
            n.vx = V_X; n.vt = V_T2; n.out = V_T2; n.mode = OUT_ADD;
            if (tree_pass(n, Tb, L0, L0, Tb.maxlev, false,
                          [&](NBuilder& nb, int64_t c) { bwd_child(nb, Tb, sEb, c); })) {
                downL0 = L0;
                downIdx = int(p.npasses.size()) - 1;
            } else {
                drop_n();
            }
        }
        std::vector<Stage>& lv = p.stages_mr[op];
        std::vector<Stage>& sw = p.stages[op];
        lv = {leaves_in};
        sw = {leaves_in};
        if (upIdx >= 0) sw.push_back({1, upIdx});
        for (int lev = Tf.maxlev - 1; lev >= 0; --lev) {
            if (up[size_t(lev)] < 0) continue;
            lv.push_back({1, up[size_t(lev)]});
            if (upIdx < 0 || lev < upL0) sw.push_back({1, up[size_t(lev)]});
        }
        lv.push_back(mid);
        sw.push_back(mid);
        for (int lev = 0; lev < Tb.maxlev; ++lev) {
            if (down[size_t(lev)] < 0) continue;
            lv.push_back({1, down[size_t(lev)]});
            if (downIdx < 0 || lev + 1 < downL0) sw.push_back({1, down[size_t(lev)]});
        }
        if (downIdx >= 0) sw.push_back({1, downIdx});
        lv.insert(lv.end(), tail.begin(), tail.end());
        sw.insert(sw.end(), tail.begin(), tail.end());
        if (upIdx < 0 && downIdx < 0) lv.clear();   // the same stages
    };

    // ---- op N
    fwd_leaves(add_tt("h2_fwd_leaves"), Cc, tc, cbl, sCB);
    const Stage n_leaves{2, int(p.ttpasses.size()) - 1};
    {   // couplings: every row cluster of positive rank is written (zero without blocks)
        NPass& c = add_n("h2_coupling");
        c.vx = V_X; c.vt = V_T; c.out = V_T2; c.mode = OUT_SET;
        NBuilder nbld(c, st);
        for (int64_t t = 0; t < R.n; ++t) {
            if (R.c[t].rank == 0) continue;
            const int64_t kr = R.c[t].rank;
            for (int64_t r0 = 0, piece = 0; r0 < kr; r0 += TILE, ++piece) {
                const int64_t rows = std::min<int64_t>(TILE, kr - r0);
                nbld.begin(rows);
                for (int64_t i : lr_by_row[size_t(t)])
                    nbld.slab(sS[size_t(i)][size_t(piece)], VEC_T | uint32_t(Cc.off[size_t(d.blocks[i].col_basis)]));
                nbld.end(uint32_t(R.off[size_t(t)] + r0), rows, true);
            }
        }
        nbld.finish();
    }
    const Stage n_coupling{1, int(p.npasses.size()) - 1};
    bwd_leaves(add_n("h2_bwd_leaves_Dx"), R, tr, rbl, sRB, true);
    const Stage n_out{1, int(p.npasses.size()) - 1};
    compose(HLRC_OP_N, Cc, sETC, R, sER, n_leaves, n_coupling, {n_out});
    if (g_knobs.side_dense(2)) {
        // the one-vector product with the near field on a side stream: y +=
        // alpha D x per row tile first, the leaf bases' V_t y^_t after the
        // backward transfers
        NPass& dx = add_n("h2_Dx");
        dx.vx = V_X; dx.vt = V_T2; dx.out = V_Y; dx.mode = OUT_ADD_ALPHA;
        {
            NBuilder nbld(dx, st);
            std::vector<size_t> posD(static_cast<size_t>(nb), 0);
            for (int64_t q = 0; q < tr.n(); ++q) {
                nbld.begin(tr.size(q));
                for (int64_t i : rdl[size_t(q)]) nbld.slab(sD[size_t(i)][posD[size_t(i)]++], uint32_t(d.blocks[i].col0));
                nbld.end(uint32_t(tr.lo(q)), tr.size(q), false);
            }
            nbld.finish();
        }
        const int dxi = int(p.npasses.size()) - 1;
        bwd_leaves(add_n("h2_bwd_leaves"), R, tr, rbl, sRB, false);
        const Stage lu{1, int(p.npasses.size()) - 1};
        std::vector<Stage>& nf = p.stages_nf[HLRC_OP_N];
        nf = {Stage{1, dxi, 1}};
        p.nf_multi = g_knobs.near_field == 2;
        for (const Stage& sg : p.stages[HLRC_OP_N])
            nf.push_back(sg.kind == n_out.kind && sg.idx == n_out.idx ? lu : sg);
    }

    // ---- op C: the trees exchanged
    fwd_leaves(add_tt("h2_fwd_leaves"), R, tr, rbl, sRB);
    const Stage c_leaves{2, int(p.ttpasses.size()) - 1};
    {   // couplings transposed: y^_s = sum_t S_ts^T x^_t (unit T-form; every
        // column cluster of positive rank is written)
        p.tpasses.emplace_back();
        p.names[0].push_back("h2_couplingT");
        TPass& c = p.tpasses.back();
        c.in = V_T; c.out = V_T2; c.mode = OUT_SET;
        TBuilder tb(c);
        for (int64_t s = 0; s < Cc.n; ++s) {
            if (Cc.c[s].rank == 0) continue;
            std::vector<TSlab> sl;
            for (int64_t i : lr_by_col[size_t(s)]) {
                const hlrc_uniform_block& b = d.blocks[i];
                const int64_t kr = R.c[b.row_basis].rank;
                for (int64_t r0 = 0, piece = 0; r0 < kr; r0 += TILE, ++piece) {
                    const int64_t rows = std::min<int64_t>(TILE, kr - r0);
                    sl.push_back({uint64_t(st.slab_elem_off(sS[size_t(i)][size_t(piece)])),
                                  uint32_t(R.off[size_t(b.row_basis)] + r0), uint16_t(rows), uint16_t(pad_rows(rows))});
                }
            }
            tb.add(uint32_t(Cc.off[size_t(s)]), Cc.c[s].rank, sl);
        }
        tb.finish();
    }
    const Stage c_coupling{0, int(p.tpasses.size()) - 1};
    bwd_leaves(add_n("h2_bwd_leaves"), Cc, tc, cbl, sCB, false);
    const Stage c_out{1, int(p.npasses.size()) - 1};
    plan_dense_transposed(add_tt("h2_DtX"), st, tr, tc, rdl, sD, [&](int64_t i, int64_t& c0, int64_t& nc) {
        c0 = d.blocks[i].col0;
        nc = d.blocks[i].ncols;
    });
    const Stage c_dense{2, int(p.ttpasses.size()) - 1};
    compose(HLRC_OP_C, R, sETR, Cc, sEC, c_leaves, c_coupling, {c_out, c_dense});
    p.stages[HLRC_OP_T].clear();   // as uniform-H: no transposed product
    for (const TTPass& tp : p.ttpasses)
        if (tp.npart >= (int64_t(1) << 32)) return fail(HLRC_ERR_SHAPE, "partial array exceeds 2^32 entries");

    if (hlrc_status vs = validate_plan(p); vs != HLRC_OK) return vs;

    // accounting: stored bytes (leaf bases, transfers, couplings, dense) plus
    // the vectors, and GEMV flops (utils/flops.hh:41-42)
    double flops = 0, mbytes = 0;
    for (int side = 0; side < 2; ++side) {
        const Tree& T = side == 0 ? R : Cc;
        for (int64_t t = 0; t < T.n; ++t) {
            const hlrc_h2_cluster& c = T.c[t];
            if (c.rank == 0) continue;
            if (T.leaf(t)) { flops += flops_gemv(double(c.size), c.rank); mbytes += 8.0 * c.rank * double(c.size); }
            if (t != 0 && T.c[c.parent].rank > 0) {
                flops += flops_gemv(c.rank, T.c[c.parent].rank);
                mbytes += 8.0 * c.rank * T.c[c.parent].rank;
            }
            p.max_rank = std::max(p.max_rank, c.rank);
        }
    }
    for (int64_t i = 0; i < nb; ++i) {
        const auto& b = d.blocks[i];
        if (b.kind == HLRC_LEAF_DENSE) {
            ++p.n_dense;
            flops += flops_gemv(double(b.nrows), double(b.ncols));
            mbytes += 8.0 * double(b.nrows) * double(b.ncols);
        } else {
            ++p.n_lowrank;
            const double kr = R.c[b.row_basis].rank, kc = Cc.c[b.col_basis].rank;
            flops += flops_gemv(kr, kc);
            mbytes += 8.0 * kr * kc;
        }
    }
    p.matrix_bytes = int64_t(mbytes);
    p.algorithmic_bytes = int64_t(mbytes + 8.0 * double(d.ncols) + 8.0 * double(d.nrows));
    p.flops = int64_t(flops);
    return HLRC_OK;
}

}  // namespace hlrc

// Row partition of an H-matrix for one product shared by several processes:
// candidate cuts are the rows no leaf straddles; cut k is the candidate
// whose preceding leaves' stored bytes are closest to k/parts of the total
// (the last of equally close ones).  No counterpart in HLR's product.
extern "C" hlrc_status hlrc_row_cuts(const hlrc_h_desc* desc, int parts, int64_t* cuts) {
    using namespace hlrc;
    clear_error();
    if (!desc || !cuts || parts < 1) return fail(HLRC_ERR_ARG, "hlrc_row_cuts: null argument or parts < 1");
    const int64_t n = desc->nrows;
    if (n < 0 || desc->nblocks < 0 || (desc->nblocks > 0 && !desc->blocks))
        return fail(HLRC_ERR_ARG, "hlrc_row_cuts: bad descriptor");
    std::vector<int64_t> cover(size_t(n) + 2, 0);
    std::vector<double> done(size_t(n) + 1, 0.0);   // bytes of the leaves ending at a row
    for (int64_t i = 0; i < desc->nblocks; ++i) {
        const hlrc_block& b = desc->blocks[i];
        const int64_t r0 = b.row0, r1 = b.row0 + b.nrows;
        if (r0 < 0 || b.nrows < 0 || r1 > n) return fail(HLRC_ERR_SHAPE, "hlrc_row_cuts: block %lld outside the rows",
                                                          (long long)i);
        if (r1 - r0 > 1) {
            ++cover[size_t(r0) + 1];
            --cover[size_t(r1)];
        }
        done[size_t(r1)] += b.kind == HLRC_LEAF_DENSE ? 8.0 * double(b.nrows) * double(b.ncols)
                                                      : 8.0 * double(b.rank) * double(b.nrows + b.ncols);
    }
    std::vector<int64_t> cand;
    std::vector<double> prefix;
    int64_t run = 0;
    double acc = 0.0;
    for (int64_t c = 0; c <= n; ++c) {
        run += cover[size_t(c)];
        acc += done[size_t(c)];
        if (run == 0) {
            cand.push_back(c);
            prefix.push_back(acc);
        }
    }
    const double total = prefix.empty() ? 0.0 : prefix.back();
    cuts[0] = 0;
    size_t j = 0;
    for (int k = 1; k < parts; ++k) {
        const double target = total * k / parts;
        while (j + 1 < cand.size() && std::fabs(prefix[j + 1] - target) <= std::fabs(prefix[j] - target)) ++j;
        cuts[k] = std::max(cuts[k - 1], cand.empty() ? int64_t(0) : cand[j]);
    }
    cuts[parts] = n;
    return HLRC_OK;
}
