// Host-side flattening of an H-matrix / uniform-H descriptor into the slab
// layout and the work lists of the device passes (see layout.hpp).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "hlrc.h"
#include "layout.hpp"

namespace hlrc {

// Where a pass reads its vectors from / writes its result to.  The device
// code binds these names to pointers at launch time.
enum VecName : int {
    V_X = 0,      // the caller's x
    V_Y = 1,      // the caller's y
    V_T = 2,      // workspace coefficients t (H) / ux (uniform)
    V_T2 = 3,     // workspace coefficients uy (uniform)
};

// How a pass writes its outputs.
enum OutMode : int {
    OUT_SET = 0,        // out = s            (coefficients)
    OUT_ADD_ALPHA = 1,  // out += alpha * s   (y)
    OUT_ADD = 2,        // out += s           (H^2: coefficients passed down the tree)
};

// A chunk of stored matrix data as the planner sees it, before it is
// encoded into the device descriptor of the plan's precision: <= 8 columns
// of one slab, all in one storage format.
struct GChunk {
    uint64_t byte_off;     // offset of the chunk's first column in the store
    uint32_t vo;           // N-form: vector offset (| VEC_T); TT-form: output / partial offset
    uint16_t nc;           // columns
    uint8_t fmt;           // StoreFmt
    uint8_t flags;         // TT_DIRECT for tile T-form chunks; GC_PACK2 (planner only)
    float scale;           // value = stored * scale (1 for unscaled formats)
};
// planner flag: this chunk is the second part of a pack with the chunk before it
constexpr uint8_t GC_PACK2 = 0x80;

struct TPass {
    std::vector<TSlab> slabs;
    std::vector<TUnit> units;      // ordered by column class, then cost
    int cls_begin[4] = {0, 0, 0, 0};  // units of class c: [cls_begin[c], cls_begin[c+1]); classes nc<=8,16,32
    std::vector<TGroup> groups;    // outputs with several units
    uint32_t nslots = 0;
    int in = V_X, out = V_T, mode = OUT_SET;
    int64_t bytes = 0;             // stored bytes streamed by the pass (with padding)
    int64_t alg_bytes = 0;         // unpadded matrix bytes + vector reads/writes
    bool empty() const { return units.empty(); }
};

// N-form and tile-T-form passes keep one segment list per storage format:
// a tile's chunks are grouped by format, and each format runs as its own
// launch (FP64, FP32, FP16, BF16 in that fixed order).
struct NPass {
    std::vector<NSeg> segs[NFMT];     // per StoreFmt, ordered by cost (descending)
    std::vector<GChunk> chunks;
    // tree sweep (H^2 transfers, FP64 only; empty: one CTA per segment).
    // Subtree b (one cluster of TREE_CLUSTER CTAs) runs the levels
    // [cta_begin[b], cta_begin[b+1]) one after the other, with a cluster
    // barrier between them; level g is the segments [tree_level[g],
    // tree_level[g+1]) of segs[FMT_F64], of which cluster rank r computes
    // [tree_part[g*(TREE_CLUSTER+1)+r], tree_part[g*(TREE_CLUSTER+1)+r+1]).
    // Segments keep the order built, and their chunks follow one another in
    // that order.  tree_seg[s]: mirror slot of segment s's first row;
    // tree_chunk[c]: the chunk's stage offset (in its owner's stage) and
    // mirror slot; subtree b copies the coefficients
    // tree_ext[tree_cta_ext[b] .. tree_cta_ext[b+1]) into its mirrors first.
    std::vector<int32_t> cta_begin, tree_level, tree_part, tree_seg, tree_cta_ext;
    std::vector<TreeChunk> tree_chunk;
    std::vector<TreeExt> tree_ext;
    int64_t tree_stage = 0, tree_mirror = 0;   // most stage doubles (one CTA) / mirror slots (one subtree)
    int tree_levels = 0, tree_segs = 0, tree_chunks = 0;   // most levels / segments / chunks of one subtree
    int tree_items = 0;                        // most chunks of one level computed by one CTA
    int vx = V_X, vt = V_T, out = V_Y, mode = OUT_ADD_ALPHA;
    int64_t bytes = 0;
    int64_t alg_bytes = 0;
};

struct TTPass {
    std::vector<TTSeg> segs[NFMT];    // per StoreFmt, ordered by cost (descending)
    std::vector<GChunk> chunks;
    std::vector<TGroup> groups;    // multi-tile outputs: partials summed in tile order
    // first level of the finish for outputs with many tiles: each entry sums
    // at most FINISH_SLOTS slots into the scratch region at the end of the
    // partial array, which the entry's final group in `groups` then reads
    std::vector<TGroup> groups1;
    int64_t npart = 0;             // partial array length (doubles), scratch region included
    int in = V_X, out = V_T, mode = OUT_SET;
    int64_t bytes = 0, alg_bytes = 0;
};

// The one-pass 64-vector product of a 16-bit H store (op N): the
// column-cluster T-form units and their tables, the finish groups of
// clusters cut into pieces, and the static exponents of t's split rows
// (c_i = ceil(log2 ||V(:,i)||_1), so |t_i| 2^g / 2^c_i <= 2^14 whenever
// max |x| 2^g < 2^14).  Empty when the plan has no such product.
struct WidePlan {
    std::vector<WTUnit> units;     // by cost, descending
    std::vector<WTBlk> blks;
    std::vector<uint32_t> slabs;
    std::vector<WTTile> tiles;
    std::vector<TGroup> groups;    // per block of a cut cluster: sums its pieces' partials into t
    int64_t npart = 0;             // partial entries (WIDE_RHS FP32 values each)
    std::vector<int8_t> t_exp;     // per t entry
    bool empty() const { return units.empty(); }
};

// One stage of a product: exactly one of the passes is used.
struct Stage {
    int kind;                      // 0 = T-form (units), 1 = N-form, 2 = tile T-form
    int idx;                       // index into Plan::tpasses / npasses / ttpasses
    // 1: launched on the workspace's side stream at the start of the product
    // (an N-form pass that writes y and reads only x and the store); the
    // first stage after it that writes y waits for it
    int side = 0;
};

// One column block of an FP64 store whose source leaves are in device
// memory: nc columns of `rows` doubles from src (leading dimension lds) to
// store byte offset dst (leading dimension ldc; rows past `rows` stay zero).
struct DevCopy {
    uint64_t dst;
    const double* src;
    int64_t lds;
    int32_t rows, nc, ldc, pad;
};
static_assert(sizeof(DevCopy) == 40, "DevCopy is 40 bytes");

struct Plan {
    int kind = 0;                  // 0 = H, 1 = uniform-H, 2 = H^2
    int precision = HLRC_PREC_F64;
    int64_t nrows = 0, ncols = 0;
    std::vector<uint8_t> store;    // slab storage (FP64, or per-chunk formats)
    // device-resident leaves (FP64): the store is filled on the device by
    // these copies instead of from `store`, which stays empty
    bool dev_src = false;
    int64_t dev_store_bytes = 0;
    std::vector<DevCopy> dev_copies;
    int64_t store_size() const { return dev_src ? dev_store_bytes : int64_t(store.size()); }
    int64_t n_t = 0, n_t2 = 0;     // workspace vector lengths (per rhs)
    std::vector<TPass> tpasses;
    std::vector<NPass> npasses;
    std::vector<TTPass> ttpasses;
    std::vector<Stage> stages[3];  // per op (N, T, C); empty = unsupported
    std::vector<Stage> stages_mr[3];  // multi-vector products when they differ (H^2: level passes, no tree sweeps)
    // one-vector products with the near field on a side stream
    // (hlrc_options.near_field): replaces stages[op] there when not empty
    std::vector<Stage> stages_nf[3];
    bool nf_multi = false;         // multi-vector products take stages_nf too (near_field = 2 asked for)
    // accounting (per product, one rhs)
    int64_t n_dense = 0, n_lowrank = 0, n_row_tiles = 0, n_col_tiles = 0;
    int64_t matrix_bytes = 0, algorithmic_bytes = 0, flops = 0;
    int32_t max_rank = 0;
    int64_t fmt_bytes[NFMT] = {};  // stored bytes per StoreFmt (accounting of mixed precision)
    // profile names per pass (static strings), per stage kind; empty = the
    // fixed names of kinds 0 and 1
    std::vector<const char*> names[3];
    WidePlan wide;                 // 16-bit H stores: the 64-vector op N product
};

// Returns HLRC_OK or an error (message recorded via fail()).  expected_area
// is the number of entries the leaves must cover (< 0: nrows * ncols; a
// batch passes the sum over its members).
hlrc_status plan_h(const hlrc_h_desc& d, const hlrc_options& o, Plan& p, double expected_area = -1.0);
hlrc_status plan_uniform(const hlrc_uniform_desc& d, const hlrc_options& o, Plan& p);
hlrc_status plan_h2(const hlrc_h2_desc& d, const hlrc_options& o, Plan& p);

}  // namespace hlrc
