// Flattened device layout of an H-matrix / uniform-H matrix.
//
// Every matrix that takes part in the product (dense leaf D, low-rank factor
// U or V, cluster basis V_t, coupling S) is cut into *slabs*: the rows that
// fall into one output tile (a leaf cluster of <= 64 indices), stored
// column-major and contiguous with a leading dimension padded to 16 bytes.
//
// Two generic batched GEMV forms cover all stages of the product:
//
//  N-form  y_tile (+)= alpha * sum_chunks  A_chunk * v_chunk
//          one CTA per output tile ("segment"); the tile's column chunks
//          (<= NCHUNK columns of one slab each) are spread over the CTA's
//          warps; each lane owns two rows; warps are combined in a fixed
//          order, so the result is deterministic (no atomics).
//          Used for: U * t (per row tile), D * x, V_t * uy, S * ux.
//
//  T-form  out[0:nc] = sum_slabs  A_slab(:, c0:c0+nc)^T * x_slab
//          one warp per work unit (a run of slabs of one block and <= 32
//          columns); lanes own two rows; the per-lane column partials are
//          combined by a butterfly transpose-reduction.  Units of one output
//          are summed by a finish pass in fixed order (or written directly
//          when an output has a single unit).
//          Used for: V^T x (op N), U^T x (op T), D^T x (op T), V_s^T x.
#pragma once

#include <cstdint>

namespace hlrc {

constexpr int TILE = 64;          // max rows of an output tile / slab
constexpr int NCHUNK = 8;         // columns per N-form chunk
constexpr int TCOLS = 8;          // columns per T-form unit (register-light: 8 partials per lane)
constexpr uint32_t VEC_T = 0x80000000u;  // v_off flag: vector lives in the t array

struct NChunk {            // N-form work item: columns [0,nc) of one slab
    uint64_t a_off;        // element offset of the chunk's first column
    uint32_t v_off;        // offset of the vector entries (| VEC_T: in t)
    uint16_t nc;           // columns (<= NCHUNK)
    uint16_t sidx;         // scale index slot (reduced precision), unused for FP64
};
static_assert(sizeof(NChunk) == 16, "NChunk must be 16 bytes");

struct NSeg {              // N-form output tile
    uint32_t cb, ce;       // chunk range
    uint32_t out;          // offset of the tile's first output entry
    uint16_t rows;         // rows of the tile (<= 64)
    uint16_t ld;           // leading dimension of all slabs of this tile
};
static_assert(sizeof(NSeg) == 16, "NSeg must be 16 bytes");

struct TSlab {             // T-form input slab
    uint64_t a_off;        // element offset of the slab's column 0
    uint32_t v_off;        // offset of the slab's first row in the input vector
    uint16_t rows;         // rows (<= 64)
    uint16_t ld;           // leading dimension (rows padded)
};
static_assert(sizeof(TSlab) == 16, "TSlab must be 16 bytes");

enum : uint8_t {
    TU_DIRECT = 1,         // single unit of its output: write the result itself
};

struct TUnit {             // T-form work unit (one warp)
    uint32_t sb, se;       // slab range
    uint32_t out;          // DIRECT: output offset; else partial slot (x32)
    uint16_t c0;           // first column of the unit within the slabs
    uint8_t nc;            // columns (<= 32)
    uint8_t flags;
};
static_assert(sizeof(TUnit) == 16, "TUnit must be 16 bytes");

struct TGroup {            // output of several T-form units, summed in order
    uint32_t slot0;        // unit passes: partial slots [slot0, slot0+nslots), 32 doubles each;
                           // tile passes: partials at slot0 + i*nc + j, i < nslots
    uint32_t nslots;
    uint32_t out;          // output offset
    uint32_t nc;           // columns
};
static_assert(sizeof(TGroup) == 16, "TGroup must be 16 bytes");

// Tile T-form ("TT"): one CTA per input tile (<= 64 rows of x); the tile's
// slabs are contiguous in the store.  Every chunk (<= TCOLS columns of one
// slab) is reduced on its own and written to its output or partial slot.
enum : uint16_t {
    TT_DIRECT = 1,         // chunk output is final (object has a single tile)
};

struct TTChunk {
    uint64_t a_off;        // element offset of the chunk's first column
    uint32_t out;          // DIRECT: output offset; else offset in the partial array
    uint16_t nc;           // columns (<= TCOLS)
    uint16_t flags;
};
static_assert(sizeof(TTChunk) == 16, "TTChunk must be 16 bytes");

struct TTSeg {
    uint32_t cb, ce;       // chunk range
    uint32_t v_off;        // first row of the tile in the input vector
    uint16_t rows;         // rows of the tile (<= 64)
    uint16_t ld;           // leading dimension of all slabs of the tile
};
static_assert(sizeof(TTSeg) == 16, "TTSeg must be 16 bytes");

// ------------------------------------------------------ reduced precision
// Storage formats of a chunk.  Scaled formats store value / scale; the
// scale (one FP32 per chunk = per block, tile and <= 8 columns) is folded
// into the chunk's partial sum.
enum StoreFmt : uint8_t {
    FMT_F64 = 0,
    FMT_F32 = 1,
    FMT_F16 = 2,     // IEEE binary16, scaled
    FMT_BF16 = 3,    // bfloat16, scaled
    FMT_I16 = 4,     // 16-bit integer (block floating point), scaled; stored offset-binary (v + 2^15)
    FMT_I24 = 5,     // 24-bit integer (block floating point, |v| < 2^22), scaled; offset-binary
                     // u = v + 2^22 stored per column as ld 16-bit high parts (u >> 8), then ld
                     // 8-bit low parts
};
constexpr int NFMT = 6;   // number of storage formats

inline constexpr int fmt_bytes(int f) {
    return f == FMT_F64 ? 8 : (f == FMT_F32 ? 4 : (f == FMT_I24 ? 3 : 2));
}

struct QNChunk {           // N-form chunk of a reduced-precision store
    uint32_t a16;          // byte offset / 16 of the chunk's first column
    uint32_t v_off;        // vector offset (| VEC_T)
    float scale;
    uint16_t nc;
    uint8_t fmt;
    uint8_t pad;
};
static_assert(sizeof(QNChunk) == 16, "QNChunk must be 16 bytes");

struct QTTChunk {          // tile T-form chunk of a reduced-precision store
    uint32_t a16;
    uint32_t out;          // DIRECT: output offset; else partial offset
    float scale;
    uint16_t nc;
    uint8_t fmt;
    uint8_t flags;
};
static_assert(sizeof(QTTChunk) == 16, "QTTChunk must be 16 bytes");

// Reduced-precision work items: two chunks of one tile and format whose
// columns together fit the format's 4 KB capacity (16 FP32 / 32 16-bit
// columns), processed as one (second part empty when nc == 0).  Low-rank
// blocks split into FP32 and FP16 column runs would otherwise fill chunks
// only about half.
struct QNPack { QNChunk p[2]; };
struct QTTPack { QTTChunk p[2]; };
static_assert(sizeof(QNPack) == 32 && sizeof(QTTPack) == 32, "packs must be 32 bytes");

// One output tile of a reduced-precision N-form pass with the packs of both
// of its formats: FP32 packs [cb32, ce32) and packs of the store's 16-bit
// format [cb16, ce16), each range possibly empty.
struct NSeg2 {
    uint32_t cb32, ce32, cb16, ce16;
    uint32_t out;          // offset of the tile's first output entry
    uint16_t rows;         // rows of the tile (<= 64)
    uint16_t ld32, ld16;   // leading dimensions of the two formats
    uint16_t pad0;
    uint32_t pad1;
};
static_assert(sizeof(NSeg2) == 32, "NSeg2 is 32 bytes");

// ------------------------------------------------ multi-RHS column streams
// The reduced-precision stores are laid out so that the chunks of one format
// that one pass segment (tile) visits are contiguous: the multi-RHS kernels
// stream a segment as one run of columns (column j at a16*16 + j*ld*element
// bytes) with one table entry per column.
struct MSeg {
    uint32_t a16;          // byte offset / 16 of the segment's first column
    uint32_t ncols;        // columns in the run
    uint32_t col0;         // first entry of the column table
    uint32_t vo;           // N-form: first output row; tile T-form: first input row
    uint16_t rows;         // rows of the tile (<= 64)
    uint16_t ld;           // leading dimension of every column
    uint32_t pad;
};
static_assert(sizeof(MSeg) == 24, "MSeg is 24 bytes");

constexpr uint32_t MC_DIRECT = 0x80000000u;   // tile T-form column table: output, not partial slot
// Longest run of partial slots one finish lane sums: longer outputs are
// summed in two levels (runs of at most FINISH_SLOTS slots first).
constexpr uint32_t FINISH_SLOTS = 16;
// Tree sweeps (H^2 transfers): one thread-block cluster of TREE_CLUSTER
// CTAs (TREE_WARPS warps each) per subtree.  Each level's segments are split
// between the cluster's CTAs; a CTA stages the matrix data of its own
// segments' chunks (`stage` doubles), keeps a mirror of the subtree's
// coefficients (`mirror` doubles, the same layout in every CTA), one
// mbarrier per level, the subtree's segment and chunk descriptors, its
// level and run bounds, and the partial sums of its chunks of one level
// (`items` x TILE doubles): at most
// TREE_SMEM bytes (tree_smem_bytes).  Subtrees are rooted at the first level
// with at least TREE_MIN_SUBTREES clusters, or deeper when one does not fit.
constexpr int TREE_CLUSTER = 4;
constexpr int TREE_WARPS = 16;
constexpr int TREE_SMEM = 200 * 1024;
constexpr int TREE_MIN_SUBTREES = 32;
inline constexpr int64_t tree_smem_bytes(int64_t stage, int64_t mirror, int64_t levels, int64_t segs, int64_t chunks,
                                         int64_t items) {
    return 8 * stage + 8 * ((mirror + 1) & ~int64_t(1)) + 8 * ((levels + 1) & ~int64_t(1)) +
           20 * ((segs + 3) & ~int64_t(3)) + 24 * chunks + 8 * TILE * items + 16 * (levels + 1);
}
struct TreeChunk {         // tree entry of a chunk
    uint32_t stage;        // offset (doubles, even) of its data in its owner CTA's stage
    uint32_t mirror;       // mirror slot of its first vector entry
};
struct TreeExt {           // coefficient read from outside the CTA, copied into the mirror
    uint32_t mirror;       // mirror slot
    uint32_t v_off;        // vector offset (| VEC_T: in t)
};

struct MCol {
    uint32_t idx;          // N-form: vector entry (| VEC_T: in t); T-form: output (| MC_DIRECT) or partial
    float scale;           // the chunk's scale (1 for FP32)
};
static_assert(sizeof(MCol) == 8, "MCol is 8 bytes");

// ------------------------------------- one-pass 64-vector products (op N)
// N-form: per column of a 16-bit run, its vector entry (| VEC_T) and the
// factor f / F its staged matrix column is multiplied by (a power of two
// <= 1 as two packed 16-bit values of the store's format); F = 2^E with E in
// the run's MSeg.pad.  f = chunk scale (x columns) or chunk scale times 2^c
// of the t entry (t columns).
struct WCol {
    uint32_t idx;
    uint32_t fac;
};
static_assert(sizeof(WCol) == 8, "WCol is 8 bytes");

// Column-cluster T-form: one CTA per unit, t = V^T x of a set of low-rank
// blocks that share a column cluster, over consecutive column tiles
// [tile0, tile0 + ntiles) (a whole cluster, or a piece of a long one).  The
// blocks' V slabs of one tile are stacked as the N dimension (ncols <=
// WT_MAXN columns); the tile's split rows of x are the M operand; the
// accumulator covers all the unit's tiles, so no per-tile partials.
constexpr int WT_MAXN = 128;       // stacked columns per unit
constexpr int WT_MAXT = 32;        // tiles per unit; longer clusters are cut into pieces
constexpr int WT_MAXB = 32;        // blocks (or rank slices) per unit
struct WTUnit {
    uint32_t tile0;
    uint16_t ntiles;
    uint16_t ncols;
    uint32_t blk0;         // blocks [blk0, blk0 + nblk) of the block table
    uint32_t slab0;        // slab table: ntiles x nblk store offsets (/16), tile-major
    uint16_t nblk;
    uint16_t piece;        // piece index p of `npieces` (npieces 1: outputs are final)
    uint16_t npieces;
    uint16_t pad;
    uint32_t part0;        // pieces: partial entries of the unit's blocks (see WTBlk)
};
static_assert(sizeof(WTUnit) == 28, "WTUnit is 28 bytes");
struct WTBlk {
    uint32_t toff;         // first t entry of the block's columns
    uint16_t k;            // columns (rank, or a slice of it)
    uint16_t off;          // first stacked column of the unit
    float scale;           // the V chunks' common scale (value = stored * scale)
    uint32_t pbase;        // pieces: partial entry of piece i, column l = pbase + i * k + l
};
static_assert(sizeof(WTBlk) == 16, "WTBlk is 16 bytes");
// T-form column table of a full-tile unit (WT_MAXN entries per unit, unit
// by unit): per stacked column its output entry (t row or partial entry;
// WT_NODST for padding) and its factor: the V chunks' scale, times 2^-c of
// the t entry for final outputs (a power of two in FP32 range).
struct WCDst {
    uint32_t dst;
    float fac;
    int32_t exp;
    uint32_t pad;
};
static_assert(sizeof(WCDst) == 16, "WCDst is 16 bytes");
constexpr uint32_t WT_NODST = 0xffffffffu;   // WCDst.dst of a padding column

struct WTTile {
    uint32_t v_off;        // first x entry of the column tile
    uint16_t rows;
    uint16_t ld;           // 16-bit slab leading dimension (rows padded to 8)
};
static_assert(sizeof(WTTile) == 8, "WTTile is 8 bytes");

// 64-vector N-form of full 64-row tiles with TMA: a segment (output tile) is
// a list of stages, one per run of at most 32 columns whose vector entries
// are consecutive; the matrix columns of a stage are consecutive 128-byte
// rows of the store (srow = byte offset / 128).  Every column of the
// segment has factor 1 (the store's row-group scales), E as in MSeg.pad.
struct WSeg {
    uint32_t st0, nst;     // stages [st0, st0 + nst)
    uint32_t out;          // first output row
    int32_t E;
};
static_assert(sizeof(WSeg) == 16, "WSeg is 16 bytes");
struct WStage {
    uint32_t srow;         // first matrix column: store row of 128 bytes
    uint32_t e0;           // first vector entry (| VEC_T: in t)
    uint32_t nc;           // columns (1 .. 32)
};
static_assert(sizeof(WStage) == 12, "WStage is 12 bytes");

}  // namespace hlrc
