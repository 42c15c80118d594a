// Device handle, upload and the product entry points of the hlrc C ABI.
//
// hlrc_mvm replaces hlr::tbb::mul_vec (include/hlr/tbb/arith.hh:312-340) and
// hlr::tbb::uniform::mul_vec (include/hlr/tbb/arith_uniform.hh:36-96).  The
// CPU versions recurse over the block tree, apply each leaf into a temporary
// and add it under 64-row chunk locks (tbb/detail/arith.hh:95-175); here the
// product is a fixed sequence of 2-4 batched passes over a flattened layout,
// and every output tile is written by exactly one CTA, so the result is
// deterministic and needs no atomics.
#include <cfloat>
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <type_traits>
#include <unordered_map>
#include <vector>

#include "common.hpp"
#include "hlrc.h"
#include "kernels_bfp8.cuh"
#include "kernels_f64.cuh"
#include "kernels_mr.cuh"
#include "kernels_q.cuh"
#include "kernels_tc.cuh"
#include "kernels_wide.cuh"
#include "kernels_wtma.cuh"
#include "plan.hpp"

namespace hlrc {

struct DevTPass {
    const TUnit* units = nullptr;
    const TSlab* slabs = nullptr;
    const TGroup* groups = nullptr;
    int cls_begin[4] = {0, 0, 0, 0};
    int ngroups = 0;
    int in = V_X, out = V_T, mode = OUT_SET;
    int64_t bytes = 0, alg_bytes = 0;
    int launches() const {
        int n = ngroups > 0 ? 1 : 0;
        for (int c = 0; c < 3; ++c) n += cls_begin[c + 1] > cls_begin[c] ? 1 : 0;
        return n;
    }
};

struct DevNPass {
    const NSeg* segs[NFMT] = {};         // per StoreFmt
    int nsegs[NFMT] = {};
    const MSeg* mseg[NFMT] = {};         // multi-RHS column streams (reduced precision)
    int nmseg[NFMT] = {};
    const MCol* mcol = nullptr;
    const NSeg2* seg2 = nullptr;      // reduced precision: both formats of a tile in one CTA
    const WCol* wcol = nullptr;       // 64-vector N-form: per column of the 16-bit runs
    const WSeg* wseg = nullptr;       // 64-vector N-form with TMA: full 64-row tiles
    const WStage* wstage = nullptr;
    int nwseg = 0;
    const MSeg* mseg_cp = nullptr;    // 64-vector N-form with cp.async: the other tiles
    int nmseg_cp = 0;
    int nseg2 = 0;
    int f16 = FMT_F16;                // the store's 16-bit format
    int wide = FMT_F32;               // the store's wide format (FP32, or 24-bit for BFP)
    const void* chunks = nullptr;     // NChunk (FP64 plan) or QNChunk (reduced precision)
    int vx = V_X, vt = V_T, out = V_Y, mode = OUT_ADD_ALPHA;
    int64_t bytes = 0, alg_bytes = 0;
    // tree sweep (H^2 transfers): ncta CTAs, one cluster of TREE_CLUSTER per subtree
    TreeArgs tree{};
    int ncta = 0;
    size_t tree_smem = 0;   // dynamic shared memory of the sweep
    int launches() const {
        if (nseg2 > 0 || ncta > 0) return 1;
        int n = 0;
        for (int f = 0; f < NFMT; ++f) n += nsegs[f] > 0 ? 1 : 0;
        return n;
    }
};

struct DevTTPass {
    const TTSeg* segs[NFMT] = {};
    int nsegs[NFMT] = {};
    const MSeg* mseg[NFMT] = {};
    int nmseg[NFMT] = {};
    const MCol* mcol = nullptr;
    const void* chunks = nullptr;     // TTChunk (FP64 plan) or QTTChunk
    const TGroup* groups = nullptr;
    int ngroups = 0;
    const TGroup* groups1 = nullptr;  // first finish level (long outputs), into the partial array
    int ngroups1 = 0;
    int64_t npart = 0;
    int in = V_X, out = V_T, mode = OUT_SET;
    int64_t bytes = 0, alg_bytes = 0;
    int launches() const {
        const int n = (ngroups > 0 ? 1 : 0) + (ngroups1 > 0 ? 1 : 0);
        // reduced-precision stores: one grid for the runs of all formats
        if (nmseg[FMT_F32] + nmseg[FMT_F16] + nmseg[FMT_BF16] + nmseg[FMT_I16] + nmseg[FMT_I24] > 0) return n + 1;
        int k = n;
        for (int f = 0; f < NFMT; ++f) k += nsegs[f] > 0 ? 1 : 0;
        return k;
    }
};

// Scratch used by one product: the coefficient vectors and the partial sums
// of a one-vector product, and (when present) the same arrays as row-major
// blocks of MR_RB vectors for the multi-vector kernels.  A product reads
// every scratch entry only after writing it in the same product.
struct Workspace {
    double* t = nullptr;
    double* t2 = nullptr;
    double* part = nullptr;
    double* mr_x = nullptr;      // null: no multi-vector arrays
    double* mr_t = nullptr;
    double* mr_t2 = nullptr;
    double* mr_part = nullptr;
    // one-pass 64-vector kernels of 16-bit stores (null: none): split rows of
    // x and t, FP32 partials of long column clusters, per-vector maxima and
    // scale exponents of x
    uint32_t* w_xs = nullptr;
    uint32_t* w_ts = nullptr;
    float* w_part = nullptr;
    unsigned long long* w_xmax = nullptr;
    int* w_g = nullptr;
    // TMA views of w_xs (boxes of 16 and 64 split rows) and w_ts (16 rows)
    bool has_tm = false;
    CUtensorMap tm_x16, tm_x64, tm_t16;
    bool profile = false;        // record per-pass events in the handle's profile
    // the side stream of one-vector products whose near field runs beside the
    // low-rank passes, and the events that fork it from and join it to the
    // caller's stream (null: side stages run on the caller's stream, first)
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
};

// Side stream and events for a workspace of a handle with side stages; the
// stream does not synchronise with the legacy default stream, the events
// only order.
hlrc_status side_create(Workspace& w) {
    if (cudaStreamCreateWithFlags(&w.side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&w.ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&w.ev_join, cudaEventDisableTiming) != cudaSuccess) {
        const cudaError_t e = cudaGetLastError();
        return fail(HLRC_ERR_CUDA, "side stream: %s", cudaGetErrorString(e));
    }
    return HLRC_OK;
}
void side_destroy(Workspace& w) {
    if (w.ev_join) cudaEventDestroy(w.ev_join);
    if (w.ev_fork) cudaEventDestroy(w.ev_fork);
    if (w.side) cudaStreamDestroy(w.side);
    w.side = nullptr;
    w.ev_fork = w.ev_join = nullptr;
}
bool has_side(const std::vector<Stage>* nf) {
    for (int op = 0; op < 3; ++op)
        for (const Stage& st : nf[op])
            if (st.side) return true;
    return false;
}

struct ProfileRec {
    const char* name;
    cudaEvent_t e0, e1;
    int64_t alg_bytes;
};

}  // namespace hlrc

using namespace hlrc;

struct hlrc_hmat_s {
    int device = 0;
    int kind = 0;
    int precision = HLRC_PREC_F64;
    int64_t nrows = 0, ncols = 0;
    char* arena = nullptr;
    size_t arena_bytes = 0;
    const uint8_t* store = nullptr;
    double* ws_t = nullptr;
    double* ws_t2 = nullptr;
    double* part = nullptr;
    int64_t n_t = 0, n_t2 = 0, n_part = 0;
    std::vector<DevTPass> t;
    std::vector<DevNPass> n;
    std::vector<DevTTPass> tt;
    std::vector<Stage> stages[3];
    std::vector<Stage> stages_mr[3];   // multi-vector products, when they differ (H^2: no tree sweeps)
    std::vector<Stage> stages_nf[3];   // one-vector products with side stages, when present
    bool nf_multi = false;             // multi-vector products take stages_nf too
    Workspace side_ws;                 // the handle's side stream and events (side stages only)
    hlrc_info info{};
    // multi-RHS workspace (FP64 plans, allocated at upload when max_nrhs > 1):
    // row-major blocks of MR_RB vectors
    char* mr_arena = nullptr;
    double *mr_x = nullptr, *mr_t = nullptr, *mr_t2 = nullptr, *mr_part = nullptr;
    char* mr_tables = nullptr;   // column streams of reduced-precision stores (MSeg / MCol)
    // one-pass 64-vector products of 16-bit H stores (op N): eligibility and
    // the workspace (allocated at upload when max_nrhs > MR_RB)
    bool wide = false;
    char* w_static = nullptr;         // the column-cluster T-form tables and t's exponents
    const WTUnit* w_units = nullptr;
    const WTBlk* w_blks = nullptr;
    const uint32_t* w_slabs = nullptr;
    const WTTile* w_tiles = nullptr;
    const TGroup* w_groups = nullptr;
    const int8_t* w_texp = nullptr;
    int w_nunits = 0, w_ngroups = 0;
    int64_t w_npart = 0;
    const WTUnit* w_units_tma = nullptr;   // units whose tiles are all full: TMA kernel
    const WCDst* w_ctab = nullptr;         // their column tables (WT_MAXN entries per unit)
    int w_nunits_tma = 0;
    bool tma = false;                      // store maps valid (full-tile TMA kernels usable)
    int sms = 148;                         // multiprocessors of the device (persistent grids)
    CUtensorMap tm_s16, tm_s8;             // the store as 128-byte rows, boxes of 16 and 8 rows
    char* w_arena = nullptr;          // workspace of the handle's own 64-vector products
    Workspace wws;                    // its arrays and tensor maps (only the w_* members are used)
    // host-pointer entry point staging (hlrc_mvm_host holds host_mu while it
    // uses these and the handle's workspace)
    double* hx = nullptr;
    double* hy = nullptr;
    size_t hx_elems = 0, hy_elems = 0;
    std::mutex host_mu;
    int* dev_err = nullptr;   // device error word (bounded waits that ran out)
    // bound of the device waits and the test hook of hlrc_debug_waits
    uint64_t wait_ns = 2000000000ull;
    int wait_skip = 0;
    std::atomic<int64_t> launches{0};   // kernels launched by this handle (any thread)
    std::vector<const char*> names[3];   // per-pass profile names (empty: fixed names)
    // launch shapes picked by the autotuner (hlrc_set_tuning)
    int nform_warps = 8;      // warps per CTA, single-vector N-form
    int ttform_warps = 8;     // warps per CTA, single-vector tile T-form
    int mr_min_nrhs = 2;      // fewest vectors that take the 8-vector kernels
    int wide_min_nrhs = MR_RB + 1;   // fewest vectors that take the 64-vector kernels (when the handle has them)
    int overlap = 1;          // one-vector kernels launched with programmatic dependent launch
    int side_at = 0;          // side stages forked after this many other stages
    // profiling
    bool profiling = false;
    std::vector<ProfileRec> prof;
    int nprof = 0;
};

namespace {

// cuTensorMapEncodeTiled, from the driver through the runtime (no link
// against the driver library)
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            f = nullptr;
        }
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
    }();
    return fn;
}

// A 2-D tensor map of 16-bit elements: `rows` rows of `inner` elements,
// `row_bytes` apart; boxes of box_inner x box_rows, 128-byte swizzle, zero
// fill outside the tensor.
bool make_map(CUtensorMap* m, const void* base, uint64_t inner, uint64_t rows, uint64_t row_bytes, uint32_t box_inner,
              uint32_t box_rows) {
    const PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc || rows == 0) return false;
    const cuuint64_t dims[2] = {inner, rows};
    const cuuint64_t strides[1] = {row_bytes};
    const cuuint32_t box[2] = {box_inner, box_rows};
    const cuuint32_t estr[2] = {1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT16, 2, const_cast<void*>(base), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

struct DeviceGuard {
    int prev = -1;
    bool ok = true;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) { ok = false; return; }
        if (dev >= 0 && dev != prev) ok = cudaSetDevice(dev) == cudaSuccess;
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

#define HLRC_CUDA(call)                                                                          \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess) return fail(HLRC_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

const char* stage_name(hlrc_hmat M, int nk, int idx) {
    // names used in profiles: kind 0 = H, 1 = uniform; nk = stage kind (0 T, 1 N, 2 tile T);
    // plans with their own names (H^2) carry them per pass
    if (!M->names[nk].empty()) return M->names[nk][size_t(idx)];
    const int kind = M->kind;
    static const char* ht[] = {"tform_unused"};
    static const char* hn[] = {"nform_Ut_Dx", "nform_Vt", "nform_Dx", "nform_Ut"};
    static const char* htt[] = {"ttform_VtX", "ttform_UtX", "ttform_DtX"};
    static const char* ut[] = {"tform_coupT"};
    static const char* un[] = {"nform_coupling", "nform_bwd_row_Dx", "nform_bwd_col", "nform_Dx", "nform_bwd_row"};
    static const char* utt[] = {"ttform_fwd_col", "ttform_fwd_row", "ttform_DtX"};
    if (kind == 0) return nk == 0 ? ht[idx] : (nk == 1 ? hn[idx] : htt[idx]);
    return nk == 0 ? ut[idx] : (nk == 1 ? un[idx] : utt[idx]);
}

// Offsets of every array inside the single device arena of a handle.
struct ArenaLayout {
    size_t store = 0;
    std::vector<size_t> tu, ts, tg, nc, ttc, ttg, ttg1, n2;
    std::vector<std::array<size_t, 7>> ntree;   // per N-pass: the tree sweep's seven arrays
    std::vector<std::array<size_t, NFMT>> ns, tts;   // per pass, per StoreFmt
    size_t t = 0, t2 = 0, part = 0, err = 0, total = 0;
    size_t part_elems = 0;
};

ArenaLayout arena_layout(const Plan& p) {
    ArenaLayout L;
    size_t off = 0;
    auto take = [&](size_t bytes) { const size_t o_ = off; off = align_up(off + bytes, 256); return o_; };
    static_assert(sizeof(NChunk) == sizeof(QNChunk) && sizeof(TTChunk) == sizeof(QTTChunk),
                  "FP64 and reduced-precision chunk descriptors share one size");
    L.store = take(size_t(p.store_size()));
    uint32_t max_slots = 0;
    for (const TPass& tp : p.tpasses) {
        L.tu.push_back(take(tp.units.size() * sizeof(TUnit)));
        L.ts.push_back(take(tp.slabs.size() * sizeof(TSlab)));
        L.tg.push_back(take(tp.groups.size() * sizeof(TGroup)));
        max_slots = std::max(max_slots, tp.nslots);
    }
    for (const NPass& np : p.npasses) {
        std::array<size_t, NFMT> o{};
        for (int f = 0; f < NFMT; ++f) o[size_t(f)] = take(np.segs[f].size() * sizeof(NSeg));
        L.ns.push_back(o);
        L.nc.push_back(take(np.chunks.size() * (p.precision == HLRC_PREC_F64 ? sizeof(NChunk) : sizeof(QNPack))));
        L.n2.push_back(take(p.precision == HLRC_PREC_F64
                                ? 0
                                : (np.segs[FMT_F32].size() + np.segs[FMT_F16].size() + np.segs[FMT_BF16].size() +
                                   np.segs[FMT_I16].size() + np.segs[FMT_I24].size()) *
                                      sizeof(NSeg2)));
        L.ntree.push_back({take(np.cta_begin.size() * sizeof(int32_t)), take(np.tree_level.size() * sizeof(int32_t)),
                           take(np.tree_seg.size() * sizeof(int32_t)), take(np.tree_chunk.size() * sizeof(TreeChunk)),
                           take(np.tree_ext.size() * sizeof(TreeExt)), take(np.tree_cta_ext.size() * sizeof(int32_t)),
                           take(np.tree_part.size() * sizeof(int32_t))});
    }
    size_t part_elems = size_t(std::max<uint32_t>(1, max_slots)) * 32;
    for (const TTPass& tp : p.ttpasses) {
        std::array<size_t, NFMT> o{};
        for (int f = 0; f < NFMT; ++f) o[size_t(f)] = take(tp.segs[f].size() * sizeof(TTSeg));
        L.tts.push_back(o);
        L.ttc.push_back(take(tp.chunks.size() * (p.precision == HLRC_PREC_F64 ? sizeof(TTChunk) : sizeof(QTTPack))));
        L.ttg.push_back(take(tp.groups.size() * sizeof(TGroup)));
        L.ttg1.push_back(take(tp.groups1.size() * sizeof(TGroup)));
        part_elems = std::max(part_elems, size_t(tp.npart));
    }
    L.t = take(size_t(std::max<int64_t>(1, p.n_t)) * sizeof(double));
    L.t2 = take(size_t(std::max<int64_t>(1, p.n_t2)) * sizeof(double));
    L.part = take(part_elems * sizeof(double));
    L.err = take(sizeof(int));
    L.part_elems = part_elems;
    L.total = off;
    return L;
}

// Kernel launches of a one-vector product of `op`, counted from the plan as
// the device passes count them (the dry runs report this; an upload counts
// its device passes).
int plan_launches(const Plan& p, int op) {
    const bool f64 = p.precision == HLRC_PREC_F64;
    int n = 0;
    auto formats = [](const auto& segs) {
        int k = 0;
        for (int f = 0; f < NFMT; ++f) k += segs[f].empty() ? 0 : 1;
        return k;
    };
    for (const Stage& st : p.stages_nf[op].empty() ? p.stages[op] : p.stages_nf[op]) {
        if (st.kind == 0) {
            const TPass& t = p.tpasses[size_t(st.idx)];
            n += t.groups.empty() ? 0 : 1;
            for (int c = 0; c < 3; ++c) n += t.cls_begin[c + 1] > t.cls_begin[c] ? 1 : 0;
        } else if (st.kind == 1) {
            const NPass& q = p.npasses[size_t(st.idx)];
            const int k = formats(q.segs);
            n += !q.cta_begin.empty() ? 1 : (f64 ? k : (k > 0 ? 1 : 0));
        } else {
            const TTPass& t = p.ttpasses[size_t(st.idx)];
            const int k = formats(t.segs);
            n += (t.groups.empty() ? 0 : 1) + (t.groups1.empty() ? 0 : 1) + (f64 ? k : (k > 0 ? 1 : 0));
        }
    }
    return n;
}

void fill_info(const Plan& p, const ArenaLayout& L, hlrc_info& in) {
    std::memset(&in, 0, sizeof(in));
    for (int op = 0; op < 3; ++op) in.launches[op] = plan_launches(p, op);
    in.n_rows = p.nrows; in.n_cols = p.ncols;
    in.n_dense = p.n_dense; in.n_lowrank = p.n_lowrank;
    in.n_row_tiles = p.n_row_tiles; in.n_col_tiles = p.n_col_tiles;
    in.matrix_bytes = p.matrix_bytes;
    in.algorithmic_bytes = p.algorithmic_bytes;
    in.flops = p.flops;
    in.workspace_bytes = int64_t(L.total - L.t);
    in.device_bytes = int64_t(L.total);
    in.scratch_bytes = int64_t(sizeof(double)) * (std::max<int64_t>(1, p.n_t) + std::max<int64_t>(1, p.n_t2) +
                                                  int64_t(L.part_elems));
    in.precision = p.precision;
    in.kind = p.kind;
    in.max_rank = p.max_rank;
}

// Device descriptors of the planner's chunks: FP64 plans address the store
// in doubles (64-bit offsets), reduced-precision plans in 16-byte units and
// carry each chunk's format and scale.
// FP64 plans: one 16-byte descriptor per chunk.  Reduced-precision plans: one
// 32-byte pack per chunk or pair of chunks (GC_PACK2 marks the second part);
// pack_of[i] is the pack of chunk i, used to remap segment ranges.
std::vector<uint8_t> encode_chunks(const std::vector<GChunk>& g, bool f64, bool tt, std::vector<uint32_t>& pack_of) {
    std::vector<uint8_t> out;
    pack_of.assign(g.size(), 0);
    if (f64) {
        out.resize(g.size() * 16);
        for (size_t i = 0; i < g.size(); ++i) {
            pack_of[i] = uint32_t(i);
            if (tt) {
                const TTChunk c{g[i].byte_off / 8, g[i].vo, g[i].nc, uint16_t(g[i].flags & ~GC_PACK2)};
                std::memcpy(out.data() + 16 * i, &c, 16);
            } else {
                const NChunk c{g[i].byte_off / 8, g[i].vo, g[i].nc, 0};
                std::memcpy(out.data() + 16 * i, &c, 16);
            }
        }
        return out;
    }
    auto part = [&](size_t i, uint8_t* dst) {
        if (tt) {
            const QTTChunk c{uint32_t(g[i].byte_off / 16), g[i].vo, g[i].scale, g[i].nc, g[i].fmt,
                             uint8_t(g[i].flags & ~GC_PACK2)};
            std::memcpy(dst, &c, 16);
        } else {
            const QNChunk c{uint32_t(g[i].byte_off / 16), g[i].vo, g[i].scale, g[i].nc, g[i].fmt, 0};
            std::memcpy(dst, &c, 16);
        }
    };
    uint32_t np = 0;
    for (size_t i = 0; i < g.size(); ++i) {
        if (g[i].flags & GC_PACK2) { pack_of[i] = np - 1; continue; }
        pack_of[i] = np++;
    }
    out.assign(size_t(np) * 32, 0);
    for (size_t i = 0; i < g.size(); ++i) part(i, out.data() + 32 * pack_of[i] + ((g[i].flags & GC_PACK2) ? 16 : 0));
    return out;
}

template <typename Seg>
std::vector<Seg> remap_segs(const std::vector<Seg>& segs, const std::vector<uint32_t>& pack_of) {
    std::vector<Seg> r = segs;
    for (Seg& s : r) {
        if (s.ce > s.cb) {
            const uint32_t b = pack_of[s.cb], e = pack_of[s.ce - 1] + 1;
            s.cb = b;
            s.ce = e;
        }
    }
    return r;
}

// Column streams of one pass (MSeg): the chunks of each reduced-precision
// segment, in store order, must form one contiguous run of columns; their
// columns get one MCol entry each.
struct StreamTables {
    std::vector<MSeg> seg[NFMT];
    std::vector<MCol> col;
};

template <typename Seg, typename VoOf>
hlrc_status build_streams(const std::vector<Seg> (&segs)[NFMT], const std::vector<GChunk>& chunks, bool tt, VoOf vo_of,
                          StreamTables& out) {
    for (int f = FMT_F32; f < NFMT; ++f) {
        for (const Seg& s : segs[f]) {
            if (s.ce <= s.cb) continue;
            std::vector<uint32_t> idx(s.ce - s.cb);
            for (uint32_t k = 0; k < idx.size(); ++k) idx[k] = s.cb + k;
            std::sort(idx.begin(), idx.end(),
                      [&](uint32_t a, uint32_t b) { return chunks[a].byte_off < chunks[b].byte_off; });
            const uint64_t colb = uint64_t(s.ld) * uint64_t(fmt_bytes(f));
            uint64_t expect = chunks[idx[0]].byte_off;
            if (expect % 16 != 0) return fail(HLRC_ERR_INTERNAL, "column stream not 16-byte aligned");
            MSeg m{uint32_t(expect / 16), 0, uint32_t(out.col.size()), vo_of(s), s.rows, s.ld, 0};
            for (uint32_t c : idx) {
                const GChunk& g = chunks[c];
                if (g.byte_off != expect || g.fmt != f)
                    return fail(HLRC_ERR_INTERNAL, "segment chunks are not one contiguous column run");
                expect += colb * g.nc;
                for (uint32_t j = 0; j < g.nc; ++j) {
                    uint32_t e;
                    if (tt) {
                        const uint64_t o = uint64_t(g.vo) + j;
                        if (o >= MC_DIRECT) return fail(HLRC_ERR_SHAPE, "output index beyond 2^31");
                        e = uint32_t(o) | ((g.flags & TT_DIRECT) ? MC_DIRECT : 0u);
                    } else {
                        e = ((g.vo & ~VEC_T) + j) | (g.vo & VEC_T);
                    }
                    out.col.push_back(MCol{e, g.scale});
                }
                m.ncols += g.nc;
            }
            out.seg[f].push_back(m);
        }
    }
    if (out.col.size() >= (size_t(1) << 32)) return fail(HLRC_ERR_SHAPE, "column table beyond 2^32 entries");
    return HLRC_OK;
}

// 2^d (d <= 0) as two packed 16-bit values of the store's format; 0 below
// the format's subnormal range
uint32_t pow2_pair(int d, bool bf16) {
    uint32_t b = 0;
    if (bf16) b = d >= -126 ? uint32_t(d + 127) << 7 : (d >= -133 ? 1u << (d + 133) : 0u);
    else b = d >= -14 ? uint32_t(d + 15) << 10 : (d >= -24 ? 1u << (d + 24) : 0u);
    return b | (b << 16);
}

// The 64-vector N-form's column table of one pass (WCol) and each run's
// factor exponent E (in MSeg.pad): f = chunk scale, times 2^c of the t entry
// for t columns; E = the largest exponent of f over the run; the column's
// factor is 2^(exponent of f - E).
void wide_columns(StreamTables& tab, int f, const std::vector<int8_t>& t_exp, bool bf16, std::vector<WCol>& out) {
    out.assign(tab.col.size(), WCol{0u, 0u});
    for (MSeg& m : tab.seg[f]) {
        auto fexp = [&](const MCol& c) {
            const int es = std::ilogb(c.scale);
            return (c.idx & VEC_T) ? es + int(t_exp[size_t(c.idx & ~VEC_T)]) : es;
        };
        int E = INT32_MIN;
        for (uint32_t j = 0; j < m.ncols; ++j) E = std::max(E, fexp(tab.col[size_t(m.col0 + j)]));
        if (m.ncols == 0) E = 0;
        m.pad = uint32_t(E);
        for (uint32_t j = 0; j < m.ncols; ++j) {
            const MCol& c = tab.col[size_t(m.col0 + j)];
            out[size_t(m.col0 + j)] = WCol{c.idx, pow2_pair(fexp(c) - E, bf16)};
        }
    }
}

// The 64-vector N-form's runs of full 64-row tiles become TMA segments
// (WSeg): a stage per run of <= 32 columns with consecutive vector entries
// of one array, its matrix columns at store row a16 / 8 + column (128-byte
// rows).  A run qualifies when its tile has 64 rows, it starts on a 128-byte
// boundary, and every column's factor is 1.  The other runs stay for the
// cp.async kernel.
void wide_tma_split(const StreamTables& tab, int f, const std::vector<WCol>& wcol, bool bf16, std::vector<WSeg>& segs,
                    std::vector<WStage>& stages, std::vector<MSeg>& rest) {
    const uint32_t one = pow2_pair(0, bf16);
    for (const MSeg& m : tab.seg[f]) {
        bool ok = m.rows == TILE && m.ld == TILE && m.a16 % 8 == 0 && m.ncols > 0;
        for (uint32_t j = 0; ok && j < m.ncols; ++j) ok = wcol[size_t(m.col0 + j)].fac == one;
        if (!ok) {
            rest.push_back(m);
            continue;
        }
        WSeg w{uint32_t(stages.size()), 0u, m.vo, int32_t(m.pad)};
        uint32_t j = 0;
        while (j < m.ncols) {
            const uint32_t i0 = tab.col[size_t(m.col0 + j)].idx;
            uint32_t n = 1;
            while (j + n < m.ncols && n < 32 && tab.col[size_t(m.col0 + j + n)].idx == i0 + n) ++n;
            stages.push_back(WStage{m.a16 / 8 + j, i0, n});
            j += n;
        }
        w.nst = uint32_t(stages.size()) - w.st0;
        segs.push_back(w);
    }
}

// The stream tables of a reduced-precision plan built on the host only (the
// dry run of upload_streams behind hlrc_plan_info_*): fails where an upload
// of the plan would.
hlrc_status check_streams(const Plan& p) {
    if (p.precision == HLRC_PREC_F64) return HLRC_OK;
    const int wide_pass = !p.wide.empty() && p.stages[HLRC_OP_N].size() == 2 ? p.stages[HLRC_OP_N][1].idx : -1;
    const bool bf16 = p.precision == HLRC_PREC_BF16;
    for (size_t i = 0; i < p.npasses.size(); ++i) {
        StreamTables t;
        const hlrc_status st = build_streams(p.npasses[i].segs, p.npasses[i].chunks, false,
                                             [](const NSeg& s) { return s.out; }, t);
        if (st != HLRC_OK) return st;
        if (int(i) == wide_pass) {
            const int f = bf16 ? FMT_BF16 : FMT_F16;
            std::vector<WCol> wcol;
            std::vector<WSeg> wsegs;
            std::vector<WStage> wstages;
            std::vector<MSeg> wrest;
            wide_columns(t, f, p.wide.t_exp, bf16, wcol);
            wide_tma_split(t, f, wcol, bf16, wsegs, wstages, wrest);
        }
    }
    for (size_t i = 0; i < p.ttpasses.size(); ++i) {
        StreamTables t;
        const hlrc_status st = build_streams(p.ttpasses[i].segs, p.ttpasses[i].chunks, true,
                                             [](const TTSeg& s) { return s.v_off; }, t);
        if (st != HLRC_OK) return st;
    }
    return HLRC_OK;
}

// Builds and uploads the column streams of every N-form and tile T-form pass
// (and, for plans with a 64-vector product, that N-form's column table).
hlrc_status upload_streams(const Plan& p, hlrc_hmat_s* h) {
    std::vector<StreamTables> nt(p.npasses.size()), tt(p.ttpasses.size());
    size_t bytes = 0;
    auto take = [&](size_t b) { const size_t o = bytes; bytes = align_up(bytes + b, 256); return o; };
    std::vector<std::array<size_t, NFMT>> n_seg_off(nt.size()), t_seg_off(tt.size());
    std::vector<size_t> n_col_off(nt.size()), t_col_off(tt.size());
    // the op N N-form of a 16-bit H plan with a 64-vector product
    const int wide_pass = !p.wide.empty() && p.stages[HLRC_OP_N].size() == 2 ? p.stages[HLRC_OP_N][1].idx : -1;
    const bool bf16 = p.precision == HLRC_PREC_BF16;
    std::vector<WCol> wcol;
    std::vector<WSeg> wsegs;
    std::vector<WStage> wstages;
    std::vector<MSeg> wrest;
    size_t wcol_off = 0, wseg_off = 0, wstage_off = 0, wrest_off = 0;
    for (size_t i = 0; i < nt.size(); ++i) {
        const hlrc_status st = build_streams(p.npasses[i].segs, p.npasses[i].chunks, false,
                                             [](const NSeg& s) { return s.out; }, nt[i]);
        if (st != HLRC_OK) return st;
        if (int(i) == wide_pass) {
            const int f = bf16 ? FMT_BF16 : FMT_F16;
            wide_columns(nt[i], f, p.wide.t_exp, bf16, wcol);
            wide_tma_split(nt[i], f, wcol, bf16, wsegs, wstages, wrest);
            wcol_off = take(wcol.size() * sizeof(WCol));
            wseg_off = take(wsegs.size() * sizeof(WSeg));
            wstage_off = take(wstages.size() * sizeof(WStage));
            wrest_off = take(wrest.size() * sizeof(MSeg));
        }
        for (int f = 0; f < NFMT; ++f) n_seg_off[i][size_t(f)] = take(nt[i].seg[f].size() * sizeof(MSeg));
        n_col_off[i] = take(nt[i].col.size() * sizeof(MCol));
    }
    for (size_t i = 0; i < tt.size(); ++i) {
        const hlrc_status st = build_streams(p.ttpasses[i].segs, p.ttpasses[i].chunks, true,
                                             [](const TTSeg& s) { return s.v_off; }, tt[i]);
        if (st != HLRC_OK) return st;
        for (int f = 0; f < NFMT; ++f) t_seg_off[i][size_t(f)] = take(tt[i].seg[f].size() * sizeof(MSeg));
        t_col_off[i] = take(tt[i].col.size() * sizeof(MCol));
    }
    cudaError_t e = cudaMalloc(&h->mr_tables, std::max<size_t>(bytes, 256));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(HLRC_ERR_OOM, "multi-RHS column tables of %zu bytes: %s", bytes, cudaGetErrorString(e));
    }
    auto put = [&](size_t off, const void* src, size_t b) -> cudaError_t {
        return b ? cudaMemcpy(h->mr_tables + off, src, b, cudaMemcpyHostToDevice) : cudaSuccess;
    };
    for (size_t i = 0; i < nt.size() && e == cudaSuccess; ++i) {
        for (int f = 0; f < NFMT && e == cudaSuccess; ++f) {
            e = put(n_seg_off[i][size_t(f)], nt[i].seg[f].data(), nt[i].seg[f].size() * sizeof(MSeg));
            h->n[i].mseg[f] = reinterpret_cast<const MSeg*>(h->mr_tables + n_seg_off[i][size_t(f)]);
            h->n[i].nmseg[f] = int(nt[i].seg[f].size());
        }
        if (e == cudaSuccess) e = put(n_col_off[i], nt[i].col.data(), nt[i].col.size() * sizeof(MCol));
        h->n[i].mcol = reinterpret_cast<const MCol*>(h->mr_tables + n_col_off[i]);
        if (int(i) == wide_pass) {
            if (e == cudaSuccess) e = put(wcol_off, wcol.data(), wcol.size() * sizeof(WCol));
            if (e == cudaSuccess) e = put(wseg_off, wsegs.data(), wsegs.size() * sizeof(WSeg));
            if (e == cudaSuccess) e = put(wstage_off, wstages.data(), wstages.size() * sizeof(WStage));
            if (e == cudaSuccess) e = put(wrest_off, wrest.data(), wrest.size() * sizeof(MSeg));
            DevNPass& d = h->n[i];
            d.wcol = reinterpret_cast<const WCol*>(h->mr_tables + wcol_off);
            d.wseg = reinterpret_cast<const WSeg*>(h->mr_tables + wseg_off);
            d.wstage = reinterpret_cast<const WStage*>(h->mr_tables + wstage_off);
            d.nwseg = int(wsegs.size());
            d.mseg_cp = reinterpret_cast<const MSeg*>(h->mr_tables + wrest_off);
            d.nmseg_cp = int(wrest.size());
        }
    }
    for (size_t i = 0; i < tt.size() && e == cudaSuccess; ++i) {
        for (int f = 0; f < NFMT && e == cudaSuccess; ++f) {
            e = put(t_seg_off[i][size_t(f)], tt[i].seg[f].data(), tt[i].seg[f].size() * sizeof(MSeg));
            h->tt[i].mseg[f] = reinterpret_cast<const MSeg*>(h->mr_tables + t_seg_off[i][size_t(f)]);
            h->tt[i].nmseg[f] = int(tt[i].seg[f].size());
        }
        if (e == cudaSuccess) e = put(t_col_off[i], tt[i].col.data(), tt[i].col.size() * sizeof(MCol));
        h->tt[i].mcol = reinterpret_cast<const MCol*>(h->mr_tables + t_col_off[i]);
    }
    if (e != cudaSuccess) return fail(HLRC_ERR_CUDA, "column table upload failed: %s", cudaGetErrorString(e));
    h->info.device_bytes += int64_t(bytes);
    return HLRC_OK;
}

// The tensor-core kernels use more than 48 KB of dynamic shared memory;
// the limit is raised once per device (the attribute belongs to the device
// context that is current when it is set).
hlrc_status enable_tc_smem(int dev) {
    static std::mutex mu;
    static std::vector<int> done;
    std::lock_guard<std::mutex> lock(mu);
    if (std::find(done.begin(), done.end(), dev) != done.end()) return HLRC_OK;
    HLRC_CUDA(cudaFuncSetAttribute(k_ttform_mr<FMT_F16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   tc_smem_bytes(TC_STAGE_TT, TC_STAGES_TT)));
    HLRC_CUDA(cudaFuncSetAttribute(k_ttform_mr<FMT_BF16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   tc_smem_bytes(TC_STAGE_TT, TC_STAGES_TT)));
    HLRC_CUDA(cudaFuncSetAttribute(k_nform_tc<FMT_F16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   tc_smem_bytes(TC_STAGE_N16, TC_STAGES_N16)));
    HLRC_CUDA(cudaFuncSetAttribute(k_nform_tc<FMT_BF16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   tc_smem_bytes(TC_STAGE_N16, TC_STAGES_N16)));
    HLRC_CUDA(cudaFuncSetAttribute(k_nform_d32, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   tc_smem_bytes(TC_STAGE_N32, TC_STAGES_D32)));
    HLRC_CUDA(cudaFuncSetAttribute(k_nform_bfp<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bq_smem_n(true)));
    HLRC_CUDA(cudaFuncSetAttribute(k_nform_bfp<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bq_smem_n(false)));
    HLRC_CUDA(cudaFuncSetAttribute(k_ttform_bfp<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bq_smem_t(true)));
    HLRC_CUDA(cudaFuncSetAttribute(k_ttform_bfp<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bq_smem_t(false)));
    done.push_back(dev);
    return HLRC_OK;
}

// Does the handle have 8-vector kernels?  Every store format has them (FP64
// on DMMA, FP32 columns on DMMA, 16-bit and BFP columns on FP16 MMA).
bool has_multi_kernels(hlrc_hmat) { return true; }

// Sizes of the multi-vector scratch of a handle: x, t, t2 and the partial
// sums as row-major blocks of MR_RB vectors, each array 256-byte aligned.
struct MrSizes {
    size_t nx = 0, nt = 0, nt2 = 0, np = 0, bytes = 0;
    void carve(char* base, double*& x, double*& t, double*& t2, double*& part) const {
        size_t off = 0;
        auto take = [&](size_t elems) {
            double* q = reinterpret_cast<double*>(base + off);
            off = align_up(off + elems * sizeof(double), 256);
            return q;
        };
        x = take(nx);
        t = take(nt);
        t2 = take(nt2);
        part = take(np);
    }
};

MrSizes mr_sizes(hlrc_hmat M) {
    MrSizes z;
    z.nx = size_t(std::max(M->nrows, M->ncols)) * MR_RB;
    z.nt = size_t(std::max<int64_t>(1, M->n_t)) * MR_RB;
    z.nt2 = size_t(std::max<int64_t>(1, M->n_t2)) * MR_RB;
    z.np = size_t(std::max<int64_t>(1, M->n_part)) * MR_RB;
    z.bytes = (z.nx + z.nt + z.nt2 + z.np) * sizeof(double) + 4 * 256;
    return z;
}

// Sizes of the one-pass 64-vector workspace: split rows of x (the longer
// side) and of t, FP32 partials (64 per entry), the per-vector maxima and
// scale exponents of x.
struct WideSizes {
    size_t xs = 0, ts = 0, part = 0, bytes = 0;
    void carve(char* base, Workspace& w) const {
        size_t off = 0;
        auto take = [&](size_t b) { char* q = base + off; off = align_up(off + b, 256); return q; };
        w.w_xs = reinterpret_cast<uint32_t*>(take(xs));
        w.w_ts = reinterpret_cast<uint32_t*>(take(ts));
        w.w_part = reinterpret_cast<float*>(take(part));
        w.w_xmax = reinterpret_cast<unsigned long long*>(take(WIDE_RHS * sizeof(unsigned long long)));
        w.w_g = reinterpret_cast<int*>(take(WIDE_RHS * sizeof(int)));
    }
};

WideSizes wide_sizes(hlrc_hmat M) {
    WideSizes z;
    z.xs = size_t(std::max(M->nrows, M->ncols)) * WIDE_ROWB;
    z.ts = size_t(std::max<int64_t>(1, M->n_t)) * WIDE_ROWB;
    z.part = size_t(std::max<int64_t>(1, M->w_npart)) * WIDE_RHS * sizeof(float);
    z.bytes = z.xs + z.ts + z.part + 2 * WIDE_RHS * 8 + 6 * 256;
    return z;
}

// TMA views of a workspace's split rows (x: the longer side, t: n_t rows)
void wide_ws_maps(hlrc_hmat M, Workspace& w) {
    const uint64_t nx = uint64_t(std::max(M->nrows, M->ncols)), nt = uint64_t(std::max<int64_t>(1, M->n_t));
    w.has_tm = w.w_xs && make_map(&w.tm_x16, w.w_xs, 128, nx, WIDE_ROWB, 64, 16) &&
               make_map(&w.tm_x64, w.w_xs, 128, nx, WIDE_ROWB, 64, 64) &&
               make_map(&w.tm_t16, w.w_ts, 128, nt, WIDE_ROWB, 64, 16);
}

// The store format of a 16-bit H-matrix handle whose op N product is one
// tile T-form pass (t = V^T x) followed by one N-form pass (y += alpha (U t
// + D x)) over 16-bit column runs only: the shape the 64-vector kernels
// take.  -1 otherwise.
int wide_format(hlrc_hmat M) {
    if (M->kind != 0 || (M->precision != HLRC_PREC_F16 && M->precision != HLRC_PREC_BF16) || !M->w_static) return -1;
    const std::vector<Stage>& st = M->stages[HLRC_OP_N];
    if (st.size() != 2 || st[0].kind != 2 || st[1].kind != 1) return -1;
    const DevTTPass& tp = M->tt[size_t(st[0].idx)];
    const DevNPass& np = M->n[size_t(st[1].idx)];
    const int f = M->precision == HLRC_PREC_BF16 ? FMT_BF16 : FMT_F16;
    if (tp.in != V_X || tp.out != V_T || tp.mode != OUT_SET) return -1;
    if (np.vx != V_X || np.vt != V_T || np.out != V_Y || np.mode != OUT_ADD_ALPHA || np.ncta > 0 || !np.wcol) return -1;
    for (int g = 0; g < NFMT; ++g)
        if (g != f && (tp.nmseg[g] > 0 || np.nmseg[g] > 0)) return -1;
    return f;
}

// The wide kernels use more than 48 KB of dynamic shared memory; raised once
// per device, as for the 8-vector kernels.
hlrc_status enable_wide_smem(int dev) {
    static std::mutex mu;
    static std::vector<int> done;
    std::lock_guard<std::mutex> lock(mu);
    if (std::find(done.begin(), done.end(), dev) != done.end()) return HLRC_OK;
    HLRC_CUDA(cudaFuncSetAttribute(k_nform_wtma<FMT_F16>, cudaFuncAttributeMaxDynamicSharedMemorySize, wtma_smem_n()));
    HLRC_CUDA(cudaFuncSetAttribute(k_nform_wtma<FMT_BF16>, cudaFuncAttributeMaxDynamicSharedMemorySize, wtma_smem_n()));
    HLRC_CUDA(cudaFuncSetAttribute(k_ctform_wtma<FMT_F16>, cudaFuncAttributeMaxDynamicSharedMemorySize, wtma_smem_c()));
    HLRC_CUDA(cudaFuncSetAttribute(k_ctform_wtma<FMT_BF16>, cudaFuncAttributeMaxDynamicSharedMemorySize, wtma_smem_c()));
    HLRC_CUDA(cudaFuncSetAttribute(k_ctform_wide<FMT_F16>, cudaFuncAttributeMaxDynamicSharedMemorySize, wide_smem_c()));
    HLRC_CUDA(cudaFuncSetAttribute(k_ctform_wide<FMT_BF16>, cudaFuncAttributeMaxDynamicSharedMemorySize, wide_smem_c()));
    HLRC_CUDA(cudaFuncSetAttribute(k_nform_wide<FMT_F16>, cudaFuncAttributeMaxDynamicSharedMemorySize, wide_smem_n()));
    HLRC_CUDA(cudaFuncSetAttribute(k_nform_wide<FMT_BF16>, cudaFuncAttributeMaxDynamicSharedMemorySize, wide_smem_n()));
    done.push_back(dev);
    return HLRC_OK;
}

// Checks that every column block of a device-filled store lies inside an
// allocation of device `dev` (a leaf pointer of another device or of host
// memory would make the gather kernel fault): the allocation range of a
// pointer comes from cuMemGetAddressRange, its device from
// cudaPointerGetAttributes, and confirmed ranges are cached.
using AddrRangeFn = CUresult (*)(CUdeviceptr*, size_t*, CUdeviceptr);
AddrRangeFn addr_range_fn() {
    static AddrRangeFn fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuMemGetAddressRange", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            f = nullptr;
        }
        return reinterpret_cast<AddrRangeFn>(f);
    }();
    return fn;
}

hlrc_status check_dev_copies(const std::vector<DevCopy>& cps, int dev) {
    const AddrRangeFn range = addr_range_fn();
    if (!range) return fail(HLRC_ERR_CUDA, "leaves_on_device: cuMemGetAddressRange is unavailable");
    std::vector<std::pair<uintptr_t, uintptr_t>> ok;   // confirmed [begin, end)
    for (const DevCopy& c : cps) {
        if (c.nc <= 0 || c.rows <= 0) continue;
        const uintptr_t b = reinterpret_cast<uintptr_t>(c.src);
        const uintptr_t e = b + (uintptr_t(c.lds) * uintptr_t(c.nc - 1) + uintptr_t(c.rows)) * sizeof(double);
        bool hit = false;
        for (const auto& r : ok)
            if (b >= r.first && e <= r.second) { hit = true; break; }
        if (hit) continue;
        cudaPointerAttributes at{};
        CUdeviceptr base = 0;
        size_t size = 0;
        if (cudaPointerGetAttributes(&at, c.src) != cudaSuccess || at.type != cudaMemoryTypeDevice ||
            at.device != dev || range(&base, &size, CUdeviceptr(b)) != CUDA_SUCCESS) {
            cudaGetLastError();
            return fail(HLRC_ERR_ARG, "leaves_on_device: leaf data at %p is not device memory of device %d", c.src, dev);
        }
        if (e > uintptr_t(base) + size)
            return fail(HLRC_ERR_ARG, "leaves_on_device: leaf data at %p runs past its allocation", c.src);
        ok.emplace_back(uintptr_t(base), uintptr_t(base) + size);
    }
    return HLRC_OK;
}

// The FP64 store of device-resident leaves: one warp per column block
// (DevCopy), columns one after the other, rows across the lanes.
__global__ void __launch_bounds__(256)
k_store_gather(const DevCopy* __restrict__ copies, int64_t n, char* __restrict__ store) {
    const int lane = threadIdx.x & 31;
    const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
    for (int64_t i = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; i < n; i += nw) {
        const DevCopy c = copies[i];
        double* dst = reinterpret_cast<double*>(store + c.dst);
        for (int j = 0; j < c.nc; ++j)
            for (int r = lane; r < c.rows; r += 32) dst[int64_t(j) * c.ldc + r] = c.src[int64_t(j) * c.lds + r];
    }
}

// Host copies of the leaf data of device-resident blocks (for stores that
// are planned from host data): each device allocation the blocks point into
// is copied to the host in one piece, and every block is re-pointed at the
// copy.
struct HostLeaves {
    std::vector<hlrc_block> blocks;
    std::vector<std::vector<double>> data;
};

hlrc_status leaves_to_host(const hlrc_block* blocks, int64_t nb, HostLeaves& h) {
    h.blocks.assign(blocks, blocks + nb);
    h.data.clear();
    const AddrRangeFn range = addr_range_fn();
    if (!range) return fail(HLRC_ERR_CUDA, "leaves_on_device: cuMemGetAddressRange is unavailable");
    struct Copied { uintptr_t base, end; double* host; };
    std::vector<Copied> copied;
    auto rebase = [&](const double*& ptr, int64_t ld, int64_t rows, int64_t cols) -> hlrc_status {
        if (!ptr || rows <= 0 || cols <= 0) return HLRC_OK;
        const uintptr_t b = reinterpret_cast<uintptr_t>(ptr);
        const uintptr_t e = b + uintptr_t(ld * (cols - 1) + rows) * sizeof(double);
        for (const Copied& c : copied)
            if (b >= c.base && e <= c.end) {
                ptr = reinterpret_cast<const double*>(reinterpret_cast<const char*>(c.host) + (b - c.base));
                return HLRC_OK;
            }
        CUdeviceptr base = 0;
        size_t size = 0;
        if (range(&base, &size, CUdeviceptr(b)) != CUDA_SUCCESS || e > uintptr_t(base) + size)
            return fail(HLRC_ERR_ARG, "leaves_on_device: leaf data at %p is not inside a device allocation", ptr);
        if ((uintptr_t(base) % sizeof(double)) != 0 || (b - uintptr_t(base)) % sizeof(double) != 0)
            return fail(HLRC_ERR_ARG, "leaves_on_device: leaf data at %p is not 8-byte aligned", ptr);
        h.data.emplace_back((size + sizeof(double) - 1) / sizeof(double));
        const cudaError_t ce = cudaMemcpy(h.data.back().data(), reinterpret_cast<const void*>(base), size,
                                          cudaMemcpyDeviceToHost);
        if (ce != cudaSuccess) {
            cudaGetLastError();
            return fail(HLRC_ERR_CUDA, "copying device-resident leaves to the host: %s", cudaGetErrorString(ce));
        }
        copied.push_back(Copied{uintptr_t(base), uintptr_t(base) + size, h.data.back().data()});
        ptr = reinterpret_cast<const double*>(reinterpret_cast<const char*>(copied.back().host) + (b - uintptr_t(base)));
        return HLRC_OK;
    };
    for (hlrc_block& b : h.blocks) {
        hlrc_status st = HLRC_OK;
        if (b.kind == HLRC_LEAF_DENSE) {
            st = rebase(b.D, b.ldd, b.nrows, b.ncols);
        } else if (b.rank > 0) {
            st = rebase(b.U, b.ldu, b.nrows, b.rank);
            if (st == HLRC_OK) st = rebase(b.V, b.ldv, b.ncols, b.rank);
            if (st == HLRC_OK) st = rebase(b.sv, b.rank, b.rank, 1);
        }
        if (st != HLRC_OK) return st;
    }
    return HLRC_OK;
}

// plan_h for host- or device-resident leaves: FP64 stores of device leaves
// are gathered on the device; other precisions are planned from host copies.
hlrc_status plan_h_leaves(const hlrc_h_desc& d, hlrc_options o, Plan& p, double area = -1.0) {
    if (!o.leaves_on_device || o.precision == HLRC_PREC_F64) return plan_h(d, o, p, area);
    if (d.nblocks > 0 && !d.blocks) return fail(HLRC_ERR_ARG, "blocks == NULL");
    HostLeaves hl;
    const hlrc_status st = leaves_to_host(d.blocks, std::max<int64_t>(0, d.nblocks), hl);
    if (st != HLRC_OK) return st;
    const hlrc_h_desc hd{d.nrows, d.ncols, d.nblocks, hl.blocks.data()};
    o.leaves_on_device = 0;
    return plan_h(hd, o, p, area);
}

hlrc_status upload_plan(Plan& p, const hlrc_options& o, hlrc_hmat* out) {
    auto h = std::make_unique<hlrc_hmat_s>();
    int dev = o.device;
    if (dev < 0) HLRC_CUDA(cudaGetDevice(&dev));
    DeviceGuard g(dev);
    if (!g.ok) return fail(HLRC_ERR_CUDA, "cannot select device %d", dev);
    if (o.max_nrhs > 1 && p.precision != HLRC_PREC_F64) {
        const hlrc_status st = enable_tc_smem(dev);
        if (st != HLRC_OK) return st;
    }
    h->device = dev;
    h->kind = p.kind;
    for (int k = 0; k < 3; ++k) h->names[k] = p.names[k];
    h->precision = p.precision;
    h->nrows = p.nrows;
    h->ncols = p.ncols;
    h->n_t = p.n_t;
    h->n_t2 = p.n_t2;

    const ArenaLayout L = arena_layout(p);
    h->n_part = int64_t(L.part_elems);
    const size_t o_store = L.store, o_t = L.t, o_t2 = L.t2, o_part = L.part;
    const std::vector<size_t>&o_tu = L.tu, &o_ts = L.ts, &o_tg = L.tg, &o_nc = L.nc;
    const std::vector<std::array<size_t, NFMT>>& o_ns = L.ns;
    h->arena_bytes = L.total;
    cudaError_t e = cudaMalloc(&h->arena, h->arena_bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(HLRC_ERR_OOM, "cudaMalloc of %zu bytes failed: %s", h->arena_bytes, cudaGetErrorString(e));
    }
    hlrc_hmat_s* hp = h.get();
    auto cleanup = [&]() { cudaFree(hp->arena); hp->arena = nullptr; side_destroy(hp->side_ws); };
    auto put = [&](size_t o_, const void* src, size_t bytes) -> cudaError_t {
        if (bytes == 0) return cudaSuccess;
        return cudaMemcpy(hp->arena + o_, src, bytes, cudaMemcpyHostToDevice);
    };
    const bool f64 = p.precision == HLRC_PREC_F64;
    if (!p.dev_src) {
        e = put(o_store, p.store.data(), p.store.size());
    } else {
        // leaves in device memory: the store is gathered on the device
        if (const hlrc_status cs = check_dev_copies(p.dev_copies, dev); cs != HLRC_OK) {
            cleanup();
            return cs;
        }
        e = cudaMemset(hp->arena + o_store, 0, size_t(p.dev_store_bytes));
        const size_t nc = p.dev_copies.size();
        if (e == cudaSuccess && nc > 0) {
            DevCopy* dc = nullptr;
            e = cudaMalloc(&dc, nc * sizeof(DevCopy));
            if (e == cudaSuccess) e = cudaMemcpy(dc, p.dev_copies.data(), nc * sizeof(DevCopy), cudaMemcpyHostToDevice);
            if (e == cudaSuccess) {
                const unsigned grid = unsigned(std::min<size_t>((nc + 7) / 8, size_t(148) * 16));
                k_store_gather<<<grid, 256>>>(dc, int64_t(nc), hp->arena + o_store);
                e = cudaGetLastError();
                if (e == cudaSuccess) e = cudaDeviceSynchronize();
            }
            if (dc) cudaFree(dc);
        }
    }
    for (size_t i = 0; e == cudaSuccess && i < p.tpasses.size(); ++i) {
        const TPass& tp = p.tpasses[i];
        e = put(o_tu[i], tp.units.data(), tp.units.size() * sizeof(TUnit));
        if (e == cudaSuccess) e = put(o_ts[i], tp.slabs.data(), tp.slabs.size() * sizeof(TSlab));
        if (e == cudaSuccess) e = put(o_tg[i], tp.groups.data(), tp.groups.size() * sizeof(TGroup));
        DevTPass d;
        d.units = reinterpret_cast<const TUnit*>(hp->arena + o_tu[i]);
        d.slabs = reinterpret_cast<const TSlab*>(hp->arena + o_ts[i]);
        d.groups = reinterpret_cast<const TGroup*>(hp->arena + o_tg[i]);
        std::memcpy(d.cls_begin, tp.cls_begin, sizeof(d.cls_begin));
        d.ngroups = int(tp.groups.size());
        d.in = tp.in; d.out = tp.out; d.mode = tp.mode; d.bytes = tp.bytes; d.alg_bytes = tp.alg_bytes;
        hp->t.push_back(d);
    }
    for (size_t i = 0; e == cudaSuccess && i < p.npasses.size(); ++i) {
        const NPass& np = p.npasses[i];
        DevNPass d;
        std::vector<uint32_t> pack_of;
        const std::vector<uint8_t> enc = encode_chunks(np.chunks, f64, false, pack_of);
        for (int f = 0; f < NFMT && e == cudaSuccess; ++f) {
            const std::vector<NSeg> sg = remap_segs(np.segs[f], pack_of);
            e = put(o_ns[i][size_t(f)], sg.data(), sg.size() * sizeof(NSeg));
            d.segs[f] = reinterpret_cast<const NSeg*>(hp->arena + o_ns[i][size_t(f)]);
            d.nsegs[f] = int(sg.size());
        }
        if (e == cudaSuccess) e = put(o_nc[i], enc.data(), enc.size());
        d.chunks = hp->arena + o_nc[i];
        d.vx = np.vx; d.vt = np.vt; d.out = np.out; d.mode = np.mode; d.bytes = np.bytes; d.alg_bytes = np.alg_bytes;
        if (!np.cta_begin.empty() && e == cudaSuccess) {
            if (!f64) {
                cleanup();
                return fail(HLRC_ERR_INTERNAL, "tree sweep in a reduced-precision plan");
            }
            const std::array<size_t, 7>& o = L.ntree[i];
            e = put(o[0], np.cta_begin.data(), np.cta_begin.size() * sizeof(int32_t));
            if (e == cudaSuccess) e = put(o[1], np.tree_level.data(), np.tree_level.size() * sizeof(int32_t));
            if (e == cudaSuccess) e = put(o[2], np.tree_seg.data(), np.tree_seg.size() * sizeof(int32_t));
            if (e == cudaSuccess) e = put(o[3], np.tree_chunk.data(), np.tree_chunk.size() * sizeof(TreeChunk));
            if (e == cudaSuccess) e = put(o[4], np.tree_ext.data(), np.tree_ext.size() * sizeof(TreeExt));
            if (e == cudaSuccess) e = put(o[5], np.tree_cta_ext.data(), np.tree_cta_ext.size() * sizeof(int32_t));
            if (e == cudaSuccess) e = put(o[6], np.tree_part.data(), np.tree_part.size() * sizeof(int32_t));
            TreeArgs& ta = d.tree;
            ta.cta_begin = reinterpret_cast<const int*>(hp->arena + o[0]);
            ta.level = reinterpret_cast<const int*>(hp->arena + o[1]);
            ta.seg = reinterpret_cast<const int*>(hp->arena + o[2]);
            ta.chunk = reinterpret_cast<const TreeChunk*>(hp->arena + o[3]);
            ta.ext = reinterpret_cast<const TreeExt*>(hp->arena + o[4]);
            ta.cta_ext = reinterpret_cast<const int*>(hp->arena + o[5]);
            ta.part = reinterpret_cast<const int*>(hp->arena + o[6]);
            ta.items = np.tree_items;
            ta.stage = int(np.tree_stage);
            ta.mirror = int(np.tree_mirror);
            ta.levels = np.tree_levels;
            ta.segs = np.tree_segs;
            ta.chunks = np.tree_chunks;
            d.ncta = (int(np.cta_begin.size()) - 1) * TREE_CLUSTER;
            d.tree_smem = size_t(tree_smem_bytes(np.tree_stage, np.tree_mirror, np.tree_levels, np.tree_segs,
                                                 np.tree_chunks, np.tree_items));
            if (e == cudaSuccess && d.tree_smem > 48 * 1024)
                e = cudaFuncSetAttribute(k_ntree_f64<TREE_WARPS>, cudaFuncAttributeMaxDynamicSharedMemorySize, TREE_SMEM);
        }
        if (!f64 && e == cudaSuccess) {
            // pair the FP32 and 16-bit segments of every output tile
            // the store's wide and 16-bit formats: 24-bit and 16-bit integers
            // (block floating point), or FP32 and one of FP16 / BF16
            auto has = [&](int f) { return !np.segs[f].empty(); };
            const bool bfp = has(FMT_I24) || has(FMT_I16);
            d.wide = bfp ? FMT_I24 : FMT_F32;
            d.f16 = bfp ? FMT_I16 : (has(FMT_BF16) ? FMT_BF16 : FMT_F16);
            if ((bfp && (has(FMT_F32) || has(FMT_F16) || has(FMT_BF16))) || (has(FMT_F16) && has(FMT_BF16))) {
                cleanup();
                return fail(HLRC_ERR_INTERNAL, "N-pass with an unsupported mix of formats");
            }
            const std::vector<NSeg> s32 = remap_segs(np.segs[d.wide], pack_of);
            const std::vector<NSeg> s16 = remap_segs(np.segs[d.f16], pack_of);
            std::vector<NSeg2> pairs;
            std::vector<int64_t> weight;
            std::unordered_map<uint32_t, size_t> by_out;
            for (const NSeg& g : s32) {
                by_out[g.out] = pairs.size();
                pairs.push_back(NSeg2{g.cb, g.ce, 0, 0, g.out, g.rows, g.ld, 0, 0, 0});
            }
            for (const NSeg& g : s16) {
                auto it = by_out.find(g.out);
                if (it == by_out.end()) {
                    pairs.push_back(NSeg2{0, 0, g.cb, g.ce, g.out, g.rows, 0, g.ld, 0, 0});
                } else {
                    NSeg2& q = pairs[it->second];
                    q.cb16 = g.cb; q.ce16 = g.ce; q.ld16 = g.ld;
                }
            }
            // heaviest tiles first (packs are at most 4 KB each)
            std::stable_sort(pairs.begin(), pairs.end(), [](const NSeg2& a, const NSeg2& b) {
                return (a.ce32 - a.cb32) + (a.ce16 - a.cb16) > (b.ce32 - b.cb32) + (b.ce16 - b.cb16);
            });
            e = put(L.n2[i], pairs.data(), pairs.size() * sizeof(NSeg2));
            d.seg2 = reinterpret_cast<const NSeg2*>(hp->arena + L.n2[i]);
            d.nseg2 = int(pairs.size());
        }
        hp->n.push_back(d);
    }
    for (size_t i = 0; e == cudaSuccess && i < p.ttpasses.size(); ++i) {
        const TTPass& tp = p.ttpasses[i];
        DevTTPass d;
        std::vector<uint32_t> pack_of;
        const std::vector<uint8_t> enc = encode_chunks(tp.chunks, f64, true, pack_of);
        for (int f = 0; f < NFMT && e == cudaSuccess; ++f) {
            const std::vector<TTSeg> sg = remap_segs(tp.segs[f], pack_of);
            e = put(L.tts[i][size_t(f)], sg.data(), sg.size() * sizeof(TTSeg));
            d.segs[f] = reinterpret_cast<const TTSeg*>(hp->arena + L.tts[i][size_t(f)]);
            d.nsegs[f] = int(sg.size());
        }
        if (e == cudaSuccess) e = put(L.ttc[i], enc.data(), enc.size());
        if (e == cudaSuccess) e = put(L.ttg[i], tp.groups.data(), tp.groups.size() * sizeof(TGroup));
        if (e == cudaSuccess) e = put(L.ttg1[i], tp.groups1.data(), tp.groups1.size() * sizeof(TGroup));
        d.chunks = hp->arena + L.ttc[i];
        d.groups = reinterpret_cast<const TGroup*>(hp->arena + L.ttg[i]);
        d.ngroups = int(tp.groups.size());
        d.groups1 = reinterpret_cast<const TGroup*>(hp->arena + L.ttg1[i]);
        d.ngroups1 = int(tp.groups1.size());
        d.npart = tp.npart;
        d.in = tp.in; d.out = tp.out; d.mode = tp.mode; d.bytes = tp.bytes; d.alg_bytes = tp.alg_bytes;
        hp->tt.push_back(d);
    }
    if (e == cudaSuccess) e = cudaMemset(hp->arena + L.err, 0, sizeof(int));
    if (e != cudaSuccess) {
        cleanup();
        return fail(HLRC_ERR_CUDA, "upload copy failed: %s", cudaGetErrorString(e));
    }
    // FP64 plans carry FP64 descriptors only, reduced-precision plans packs
    // only; a mix would hand one kind of kernel the other's descriptors
    for (const DevNPass& d : hp->n)
        for (int f = 0; f < NFMT; ++f)
            if (d.nsegs[f] > 0 && ((f == FMT_F64) != f64)) { cleanup(); return fail(HLRC_ERR_INTERNAL, "format mix in plan"); }
    for (const DevTTPass& d : hp->tt)
        for (int f = 0; f < NFMT; ++f)
            if (d.nsegs[f] > 0 && ((f == FMT_F64) != f64)) { cleanup(); return fail(HLRC_ERR_INTERNAL, "format mix in plan"); }
    hp->store = reinterpret_cast<const uint8_t*>(hp->arena + o_store);
    hp->ws_t = reinterpret_cast<double*>(hp->arena + o_t);
    hp->ws_t2 = reinterpret_cast<double*>(hp->arena + o_t2);
    hp->part = reinterpret_cast<double*>(hp->arena + o_part);
    hp->dev_err = reinterpret_cast<int*>(hp->arena + L.err);
    for (int op = 0; op < 3; ++op) {
        hp->stages[op] = p.stages[op];
        hp->stages_mr[op] = p.stages_mr[op];
        hp->stages_nf[op] = p.stages_nf[op];
    }
    hp->nf_multi = p.nf_multi;
    if (has_side(hp->stages_nf)) {
        if (const hlrc_status ss = side_create(hp->side_ws); ss != HLRC_OK) {
            cleanup();
            return ss;
        }
    }

    fill_info(p, L, hp->info);
    // the 8-vector kernels take FP64, FP32 and FP16/BF16 columns; block
    // floating point (BFP) stores loop the one-vector kernels instead
    if (o.max_nrhs > 1 && has_multi_kernels(hp)) {
        const MrSizes z = mr_sizes(hp);
        e = cudaMalloc(&hp->mr_arena, z.bytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            cleanup();
            return fail(HLRC_ERR_OOM, "multi-RHS workspace of %zu bytes: %s", z.bytes, cudaGetErrorString(e));
        }
        z.carve(hp->mr_arena, hp->mr_x, hp->mr_t, hp->mr_t2, hp->mr_part);
        hp->info.workspace_bytes += int64_t(z.bytes);
        hp->info.device_bytes += int64_t(z.bytes);
    }
    if (p.precision != HLRC_PREC_F64) {
        const hlrc_status st = upload_streams(p, hp);
        if (st != HLRC_OK) {
            cudaFree(hp->mr_tables);
            cudaFree(hp->mr_arena);
            cleanup();
            return st;
        }
    }
    if (!p.wide.empty()) {
        // units whose tiles are all full and whose slabs start on 128-byte
        // boundaries take the TMA kernel; they go first in the unit array
        WidePlan W = p.wide;
        {
            std::vector<WTUnit> tma_u, cp_u;
            for (const WTUnit& u : W.units) {
                bool ok = true;
                for (int t = 0; ok && t < u.ntiles; ++t) ok = W.tiles[size_t(u.tile0) + size_t(t)].rows == TILE;
                for (size_t k = 0; ok && k < size_t(u.ntiles) * u.nblk; ++k) ok = W.slabs[u.slab0 + k] % 8 == 0;
                (ok ? tma_u : cp_u).push_back(u);
            }
            hp->w_nunits_tma = int(tma_u.size());
            W.units = tma_u;
            W.units.insert(W.units.end(), cp_u.begin(), cp_u.end());
        }
        // the full-tile units' column tables (WT_MAXN entries each): output
        // entry, factor and exponent of every stacked column
        std::vector<WCDst> ctab(size_t(hp->w_nunits_tma) * WT_MAXN, WCDst{WT_NODST, 0.f, 0, 0u});
        for (int ui = 0; ui < hp->w_nunits_tma; ++ui) {
            const WTUnit& u = W.units[size_t(ui)];
            for (int j = 0; j < u.nblk; ++j) {
                const WTBlk& b = W.blks[size_t(u.blk0) + size_t(j)];
                for (int l = 0; l < b.k; ++l) {
                    WCDst& d = ctab[size_t(ui) * WT_MAXN + size_t(b.off) + size_t(l)];
                    if (u.npieces == 1) {
                        d.dst = b.toff + uint32_t(l);
                        d.exp = W.t_exp[size_t(d.dst)];
                    } else {
                        d.dst = b.pbase + uint32_t(u.piece) * b.k + uint32_t(l);
                    }
                    // chunk scale times 2^-c, kept inside the FP32 normal range
                    const double f = std::ldexp(double(b.scale), -d.exp);
                    d.fac = f == 0.0 ? 0.f : float(std::min(std::max(f, double(FLT_MIN)), double(FLT_MAX)));
                }
            }
        }
        size_t wb = 0;
        auto take = [&](size_t b) { const size_t o_ = wb; wb = align_up(wb + b, 256); return o_; };
        const size_t o_u = take(W.units.size() * sizeof(WTUnit)), o_b = take(W.blks.size() * sizeof(WTBlk)),
                     o_s = take(W.slabs.size() * sizeof(uint32_t)), o_t = take(W.tiles.size() * sizeof(WTTile)),
                     o_g = take(W.groups.size() * sizeof(TGroup)), o_e = take(W.t_exp.size()),
                     o_c = take(ctab.size() * sizeof(WCDst));
        e = cudaMalloc(&hp->w_static, std::max<size_t>(wb, 256));
        if (e == cudaSuccess) e = cudaMemcpy(hp->w_static + o_u, W.units.data(), W.units.size() * sizeof(WTUnit), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(hp->w_static + o_b, W.blks.data(), W.blks.size() * sizeof(WTBlk), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(hp->w_static + o_s, W.slabs.data(), W.slabs.size() * sizeof(uint32_t), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(hp->w_static + o_t, W.tiles.data(), W.tiles.size() * sizeof(WTTile), cudaMemcpyHostToDevice);
        if (e == cudaSuccess && !W.groups.empty())
            e = cudaMemcpy(hp->w_static + o_g, W.groups.data(), W.groups.size() * sizeof(TGroup), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(hp->w_static + o_e, W.t_exp.data(), W.t_exp.size(), cudaMemcpyHostToDevice);
        if (e == cudaSuccess && !ctab.empty())
            e = cudaMemcpy(hp->w_static + o_c, ctab.data(), ctab.size() * sizeof(WCDst), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            cudaGetLastError();
            cudaFree(hp->w_static);
            cudaFree(hp->mr_tables);
            cudaFree(hp->mr_arena);
            cleanup();
            return fail(HLRC_ERR_OOM, "64-vector tables of %zu bytes: %s", wb, cudaGetErrorString(e));
        }
        hp->w_units_tma = reinterpret_cast<const WTUnit*>(hp->w_static + o_u);
        hp->w_units = hp->w_units_tma + hp->w_nunits_tma;   // the cp.async units
        hp->w_blks = reinterpret_cast<const WTBlk*>(hp->w_static + o_b);
        hp->w_slabs = reinterpret_cast<const uint32_t*>(hp->w_static + o_s);
        hp->w_tiles = reinterpret_cast<const WTTile*>(hp->w_static + o_t);
        hp->w_groups = reinterpret_cast<const TGroup*>(hp->w_static + o_g);
        hp->w_texp = reinterpret_cast<const int8_t*>(hp->w_static + o_e);
        hp->w_ctab = reinterpret_cast<const WCDst*>(hp->w_static + o_c);
        hp->w_nunits = int(W.units.size()) - hp->w_nunits_tma;
        hp->w_ngroups = int(W.groups.size());
        hp->w_npart = W.npart;
        hp->info.device_bytes += int64_t(wb);
    }
    // the store as rows of 128 bytes for the full-tile TMA kernels
    cudaDeviceGetAttribute(&hp->sms, cudaDevAttrMultiProcessorCount, dev);
    if (hp->sms <= 0) hp->sms = 148;
    if (!p.wide.empty()) {
        const uint64_t rows = uint64_t(p.store_size()) / 128;
        hp->tma = rows > 0 && make_map(&hp->tm_s16, hp->store, 64, rows, 128, 64, 16) &&
                  make_map(&hp->tm_s8, hp->store, 64, rows, 128, 64, 8);
    }
    hp->wide = wide_format(hp) >= 0;
    if (hp->wide && o.max_nrhs > MR_RB) {
        hlrc_status st = enable_wide_smem(dev);
        const WideSizes z = wide_sizes(hp);
        if (st == HLRC_OK) {
            e = cudaMalloc(&hp->w_arena, z.bytes);
            if (e != cudaSuccess) {
                cudaGetLastError();
                st = fail(HLRC_ERR_OOM, "64-vector workspace of %zu bytes: %s", z.bytes, cudaGetErrorString(e));
            }
        }
        if (st != HLRC_OK) {
            cudaFree(hp->w_static);
            cudaFree(hp->mr_tables);
            cudaFree(hp->mr_arena);
            cleanup();
            return st;
        }
        z.carve(hp->w_arena, hp->wws);
        wide_ws_maps(hp, hp->wws);
        hp->info.workspace_bytes += int64_t(z.bytes);
        hp->info.device_bytes += int64_t(z.bytes);
    }
    for (int op = 0; op < 3; ++op) {
        int nl = 0;
        for (const Stage& st : hp->stages_nf[op].empty() ? hp->stages[op] : hp->stages_nf[op])
            nl += st.kind == 0 ? hp->t[size_t(st.idx)].launches()
                               : (st.kind == 1 ? hp->n[size_t(st.idx)].launches() : hp->tt[size_t(st.idx)].launches());
        hp->info.launches[op] = nl;
    }
    *out = h.release();
    return HLRC_OK;
}

// the handle's own workspace (hlrc_mvm, hlrc_mvm_host); only products on it
// are profiled
Workspace handle_workspace(hlrc_hmat M) {
    Workspace w;
    w.t = M->ws_t; w.t2 = M->ws_t2; w.part = M->part;
    w.mr_x = M->mr_x; w.mr_t = M->mr_t; w.mr_t2 = M->mr_t2; w.mr_part = M->mr_part;
    w.w_xs = M->wws.w_xs; w.w_ts = M->wws.w_ts; w.w_part = M->wws.w_part;
    w.w_xmax = M->wws.w_xmax; w.w_g = M->wws.w_g;
    w.has_tm = M->wws.has_tm;
    if (w.has_tm) { w.tm_x16 = M->wws.tm_x16; w.tm_x64 = M->wws.tm_x64; w.tm_t16 = M->wws.tm_t16; }
    w.profile = M->profiling;
    w.side = M->side_ws.side;
    w.ev_fork = M->side_ws.ev_fork;
    w.ev_join = M->side_ws.ev_join;
    return w;
}

double* bind(const Workspace& ws, int name, const double* x, double* y) {
    switch (name) {
        case V_X: return const_cast<double*>(x);
        case V_Y: return y;
        case V_T: return ws.t;
        default: return ws.t2;
    }
}

// Profiling events on a stream that is being captured into a CUDA graph are
// recorded as external event-record nodes, so that every replay of the graph
// records them again (a plain record during capture only orders the graph).
void prof_record(cudaEvent_t e, cudaStream_t s) {
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &st) != cudaSuccess) {
        cudaGetLastError();   // not an error of the product: clear it
        st = cudaStreamCaptureStatusNone;
    }
    if (st == cudaStreamCaptureStatusActive) cudaEventRecordWithFlags(e, s, cudaEventRecordExternal);
    else cudaEventRecord(e, s);
}

void prof_begin(hlrc_hmat M, const char* name, int64_t alg_bytes, cudaStream_t s) {
    if (!M->profiling) return;
    if (M->nprof >= int(M->prof.size())) {
        ProfileRec r{name, nullptr, nullptr, 0};
        cudaEventCreate(&r.e0);
        cudaEventCreate(&r.e1);
        M->prof.push_back(r);
    }
    M->prof[size_t(M->nprof)].name = name;
    M->prof[size_t(M->nprof)].alg_bytes = alg_bytes;
    prof_record(M->prof[size_t(M->nprof)].e0, s);
}
void prof_end(hlrc_hmat M, cudaStream_t s) {
    if (!M->profiling) return;
    prof_record(M->prof[size_t(M->nprof)].e1, s);
    ++M->nprof;
}

// warps per CTA of the single-vector kernels: the handle picks one of these
// (hlrc_tuning); each kernel is compiled for both
template <int W> using Warps = std::integral_constant<int, W>;
constexpr int DMMA_WARPS = 8;   // warps per CTA of the FP64 8-vector kernels

// Diagnostics: with HLRC_DEBUG_SYNC=1 in the environment every pass is
// followed by a stream synchronisation, and an asynchronous kernel error is
// reported with the name of the pass that raised it.
bool debug_sync() {
    static const bool on = [] {
        const char* e = std::getenv("HLRC_DEBUG_SYNC");
        return e && e[0] == '1';
    }();
    return on;
}

// A stream that is being captured is left alone: a synchronisation there
// would invalidate the capture.
bool capturing(cudaStream_t s) {
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &st) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return st != cudaStreamCaptureStatusNone;
}

#define HLRC_AFTER_LAUNCH(name)                                                                        \
    do {                                                                                               \
        if (debug_sync() && !capturing(s)) {                                                           \
            const cudaError_t e_ = cudaStreamSynchronize(s);                                           \
            if (e_ != cudaSuccess) return fail(HLRC_ERR_CUDA, "%s: %s", name, cudaGetErrorString(e_)); \
        }                                                                                              \
    } while (0)

// one right-hand side: x, y are column vectors; scratch from `ws`
// Launches k on stream s.  With `overlap` the launch carries the
// programmatic-stream-serialization attribute: the kernel may be scheduled
// while the preceding kernel of the stream still runs, and waits for it
// inside (pdl_wait) before it touches the vectors.
template <typename... P, typename... A>
cudaError_t launch_k(bool overlap, void (*k)(P...), unsigned grid, unsigned block, size_t smem, cudaStream_t s,
                     A... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = overlap ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, k, args...);
}

// Side stages (the near field) run on the workspace's side stream, forked
// from the caller's stream s0 before the first of them; the first other
// stage that writes y waits for them.  Without a side stream they run on s0
// in list order (first).
struct SideFork {
    hlrc_hmat M;
    const Workspace& ws;
    cudaStream_t s0;
    bool forked = false, joined = false;
    cudaError_t err = cudaSuccess;   // the first failed fork or join call
    void check(cudaError_t e) { if (err == cudaSuccess) err = e; }
    bool writes_y(const Stage& st) const {
        const int out = st.kind == 0 ? M->t[size_t(st.idx)].out
                                     : (st.kind == 1 ? M->n[size_t(st.idx)].out : M->tt[size_t(st.idx)].out);
        return out == V_Y;
    }
    // the stream stage st launches on
    cudaStream_t before(const Stage& st) {
        const bool on_side = st.side && ws.side;
        if (on_side && !forked) {
            check(cudaEventRecord(ws.ev_fork, s0));
            check(cudaStreamWaitEvent(ws.side, ws.ev_fork, 0));
            forked = true;
        }
        if (!st.side && forked && !joined && writes_y(st)) join();
        return on_side ? ws.side : s0;
    }
    void join() {
        check(cudaEventRecord(ws.ev_join, ws.side));
        check(cudaStreamWaitEvent(s0, ws.ev_join, 0));
        joined = true;
    }
    // after the last stage: every side stage is joined
    cudaError_t end() {
        if (forked && !joined) join();
        return err;
    }
};

// Launch order of a stage list: the other stages in list order, with the
// side stages inserted before the side_at-th of them (at most before the
// first that writes y, which waits for them).  Returns indices into stl.
const std::vector<int>& stage_order(hlrc_hmat M, const std::vector<Stage>& stl, std::vector<int>& order) {
    order.clear();
    int at = -1, m = 0;
    for (size_t i = 0; i < stl.size(); ++i) {
        if (stl[i].side) continue;
        const Stage& st = stl[i];
        const int out = st.kind == 0 ? M->t[size_t(st.idx)].out
                                     : (st.kind == 1 ? M->n[size_t(st.idx)].out : M->tt[size_t(st.idx)].out);
        if (out == V_Y) { at = m; break; }
        ++m;
    }
    at = at < 0 ? std::min(M->side_at, m) : std::min(M->side_at, at);
    auto sides = [&]() {
        for (size_t i = 0; i < stl.size(); ++i)
            if (stl[i].side) order.push_back(int(i));
    };
    m = 0;
    for (size_t i = 0; i < stl.size(); ++i) {
        if (stl[i].side) continue;
        if (m++ == at) sides();
        order.push_back(int(i));
    }
    if (at >= m) sides();
    return order;
}

hlrc_status run_single(hlrc_hmat M, const Workspace& ws, double alpha_in, int op, const double* x, double* y,
                       cudaStream_t s0) {
    // FP64 plans carry 16-byte FP64 descriptors, reduced-precision plans
    // 32-byte packs: each kind of kernel only ever sees its own kind
    const bool f64plan = M->precision == HLRC_PREC_F64;
    const bool ov = M->overlap != 0;
    cudaError_t le = cudaSuccess;   // the first failed launch
    auto L = [&](cudaError_t e) { if (le == cudaSuccess) le = e; };
    SideFork side{M, ws, s0};
    const std::vector<Stage>& stl = M->stages_nf[op].empty() ? M->stages[op] : M->stages_nf[op];
    thread_local std::vector<int> order;
    for (const int oi : stage_order(M, stl, order)) {
        const Stage& st = stl[size_t(oi)];
        const cudaStream_t s = side.before(st);
        M->launches += st.kind == 0 ? M->t[size_t(st.idx)].launches()
                                    : (st.kind == 1 ? M->n[size_t(st.idx)].launches() : M->tt[size_t(st.idx)].launches());
        if (st.kind == 0) {
            const DevTPass& tp = M->t[size_t(st.idx)];
            const double* vin = bind(ws, tp.in, x, y);
            double* vout = bind(ws, tp.out, x, y);
            const int add = tp.mode != OUT_SET;
            const double alpha = tp.mode == OUT_ADD ? 1.0 : alpha_in;   // plain adds pass coefficients down a tree
            if (ws.profile) prof_begin(M, stage_name(M, 0, st.idx), tp.alg_bytes, s);
            for (int c = 0; c < 3; ++c) {
                const int nu = tp.cls_begin[c + 1] - tp.cls_begin[c];
                if (nu <= 0) continue;
                const TUnit* u = tp.units + tp.cls_begin[c];
                const int grid = (nu + 7) / 8;
                static_assert(TCOLS == 8, "T-form units are launched with the 8-column kernel");
                const double* A = reinterpret_cast<const double*>(M->store);  // unit T-form: FP64 plans only
                if (c == 0) L(launch_k(ov, k_tform_f64<8>, grid, 256, 0, s, u, nu, tp.slabs, A, vin, vout, ws.part, alpha, add));
                else if (c == 1) L(launch_k(ov, k_tform_f64<16>, grid, 256, 0, s, u, nu, tp.slabs, A, vin, vout, ws.part, alpha, add));
                else L(launch_k(ov, k_tform_f64<32>, grid, 256, 0, s, u, nu, tp.slabs, A, vin, vout, ws.part, alpha, add));
            }
            if (tp.ngroups > 0)
                L(launch_k(ov, k_tfinish_f64, unsigned((tp.ngroups + 7) / 8), 256, 0, s, tp.groups, tp.ngroups,
                           static_cast<const double*>(ws.part), vout, alpha, add));
            if (ws.profile) prof_end(M, s);
            HLRC_AFTER_LAUNCH(stage_name(M, 0, st.idx));
        } else if (st.kind == 2) {
            const DevTTPass& tp = M->tt[size_t(st.idx)];
            if (tp.launches() == 0) continue;
            const double* vin = bind(ws, tp.in, x, y);
            double* vout = bind(ws, tp.out, x, y);
            const int add = tp.mode != OUT_SET;
            const double alpha = tp.mode == OUT_ADD ? 1.0 : alpha_in;   // plain adds pass coefficients down a tree
            if (ws.profile) prof_begin(M, stage_name(M, 2, st.idx), tp.alg_bytes, s);
            auto ttform = [&](auto wc) {
                constexpr int TW = decltype(wc)::value;
                if (f64plan && tp.nsegs[FMT_F64] > 0)
                    L(launch_k(ov, k_ttform_f64<TW>, unsigned(tp.nsegs[FMT_F64]), TW * 32, 0, s, tp.segs[FMT_F64],
                               static_cast<const TTChunk*>(tp.chunks), reinterpret_cast<const double*>(M->store), vin,
                               vout, ws.part, alpha, add));
                // reduced precision: each tile's run of columns, streamed in full
                // 4 KB iterations; FP32 and 16-bit runs in one grid
                if (!f64plan) {
                    if (tp.nmseg[FMT_I24] + tp.nmseg[FMT_I16] > 0) {   // block floating point
                        const int n24 = tp.nmseg[FMT_I24];
                        L(launch_k(ov, k_ttform_qs<TW, FMT_I24, FMT_I16>, unsigned(n24 + tp.nmseg[FMT_I16]), TW * 32, 0,
                                   s, tp.mseg[FMT_I24], n24, tp.mseg[FMT_I16], tp.mcol, M->store, vin, vout, ws.part,
                                   alpha, add));
                    } else {
                        const int n32 = tp.nmseg[FMT_F32];
                        if (tp.nmseg[FMT_BF16] > 0)
                            L(launch_k(ov, k_ttform_qs<TW, FMT_F32, FMT_BF16>, unsigned(n32 + tp.nmseg[FMT_BF16]),
                                       TW * 32, 0, s, tp.mseg[FMT_F32], n32, tp.mseg[FMT_BF16], tp.mcol, M->store, vin,
                                       vout, ws.part, alpha, add));
                        else if (n32 + tp.nmseg[FMT_F16] > 0)
                            L(launch_k(ov, k_ttform_qs<TW, FMT_F32, FMT_F16>, unsigned(n32 + tp.nmseg[FMT_F16]),
                                       TW * 32, 0, s, tp.mseg[FMT_F32], n32, tp.mseg[FMT_F16], tp.mcol, M->store, vin,
                                       vout, ws.part, alpha, add));
                    }
                }
            };
            if (M->ttform_warps == 4) ttform(Warps<4>{});
            else if (M->ttform_warps == 16) ttform(Warps<16>{});
            else ttform(Warps<8>{});
            if (ws.profile) prof_end(M, s);
            if (tp.ngroups > 0) {
                if (ws.profile) prof_begin(M, "ttfinish", tp.npart * 8, s);
                if (tp.ngroups1 > 0)   // first level: runs of slots into the scratch part of the partials
                    L(launch_k(ov, k_ttfinish_f64, unsigned((tp.ngroups1 + 7) / 8), 256, 0, s, tp.groups1, tp.ngroups1,
                               static_cast<const double*>(ws.part), ws.part, 1.0, 0));
                L(launch_k(ov, k_ttfinish_f64, unsigned((tp.ngroups + 7) / 8), 256, 0, s, tp.groups, tp.ngroups,
                           static_cast<const double*>(ws.part), vout, alpha, add));
                if (ws.profile) prof_end(M, s);
            }
            HLRC_AFTER_LAUNCH(stage_name(M, 2, st.idx));
        } else {
            const DevNPass& np = M->n[size_t(st.idx)];
            if (np.launches() == 0) continue;
            if (ws.profile) prof_begin(M, stage_name(M, 1, st.idx), np.alg_bytes, s);
            const double* vx = bind(ws, np.vx, x, y);
            const double* vt = bind(ws, np.vt, x, y);
            double* vo = bind(ws, np.out, x, y);
            const int add = np.mode != OUT_SET;
            const double alpha = np.mode == OUT_ADD ? 1.0 : alpha_in;   // plain adds pass coefficients down a tree
            auto nform = [&](auto wc) {
                constexpr int NW = decltype(wc)::value;
                if (np.ncta > 0) {   // tree sweep (FP64 plans only)
                    L(launch_k(ov, k_ntree_f64<TREE_WARPS>, unsigned(np.ncta), TREE_WARPS * 32, np.tree_smem, s,
                               np.segs[FMT_F64], static_cast<const NChunk*>(np.chunks), np.tree,
                               reinterpret_cast<const double*>(M->store), vx, vt, vo, alpha, add, M->dev_err,
                               M->wait_ns, M->wait_skip));
                    return;
                }
                if (f64plan && np.nsegs[FMT_F64] > 0)
                    L(launch_k(ov, k_nform_f64<NW>, unsigned(np.nsegs[FMT_F64]), NW * 32, 0, s, np.segs[FMT_F64],
                               static_cast<const NChunk*>(np.chunks), reinterpret_cast<const double*>(M->store), vx, vt,
                               vo, alpha, add));
                // reduced precision: one CTA per tile takes the packs of both formats
                const QNPack* qc = static_cast<const QNPack*>(np.chunks);
                if (!f64plan && np.nseg2 > 0) {
                    if (np.wide == FMT_I24)
                        L(launch_k(ov, k_nform_q<NW, FMT_I24, FMT_I16>, unsigned(np.nseg2), NW * 32, 0, s, np.seg2, qc,
                                   M->store, vx, vt, vo, alpha, add));
                    else if (np.f16 == FMT_BF16)
                        L(launch_k(ov, k_nform_q<NW, FMT_F32, FMT_BF16>, unsigned(np.nseg2), NW * 32, 0, s, np.seg2, qc,
                                   M->store, vx, vt, vo, alpha, add));
                    else
                        L(launch_k(ov, k_nform_q<NW, FMT_F32, FMT_F16>, unsigned(np.nseg2), NW * 32, 0, s, np.seg2, qc,
                                   M->store, vx, vt, vo, alpha, add));
                }
            };
            if (M->nform_warps == 4) nform(Warps<4>{});
            else if (M->nform_warps == 16) nform(Warps<16>{});
            else nform(Warps<8>{});
            if (ws.profile) prof_end(M, s);
            HLRC_AFTER_LAUNCH(stage_name(M, 1, st.idx));
        }
    }
    L(side.end());
    const cudaError_t e = le != cudaSuccess ? le : cudaGetLastError();
    if (e != cudaSuccess) return fail(HLRC_ERR_CUDA, "kernel launch failed: %s", cudaGetErrorString(e));
    return HLRC_OK;
}

// The stages of a multi-vector product: the level passes where the
// one-vector product sweeps trees.
// The 8-vector DMMA and tensor-core passes are compute-heavy, so the near
// field beside them hides nothing: multi-vector products keep the fused pass
// unless the plan asked for the side stream explicitly (near_field = 2).  On
// a uniform-H matrix (sphere, 32768 triangles, 32 vectors) the fused pass
// took 337 us against 354 us.
const std::vector<Stage>& mr_stages(hlrc_hmat M, int op) {
    if (!M->stages_mr[op].empty()) return M->stages_mr[op];
    return M->stages_nf[op].empty() || !M->nf_multi ? M->stages[op] : M->stages_nf[op];
}

// Can the product for `op` run in blocks of MR_RB right-hand sides?  Needs
// the multi-RHS workspace and no unit T-form stage (the uniform-H adjoint
// coupling runs per vector).
bool multi_rhs_ok(hlrc_hmat M, const Workspace& ws, int op, int nrhs) {
    if (nrhs < 2 || nrhs < M->mr_min_nrhs || !ws.mr_x) return false;
    for (const Stage& st : mr_stages(M, op))
        if (st.kind == 0) return false;
    return true;
}

// y := y + alpha op(M) X for nrhs column vectors, MR_RB at a time: the matrix
// is streamed once per block instead of once per vector.
hlrc_status run_multi(hlrc_hmat M, const Workspace& ws, double alpha_in, int op, const double* X, int64_t ldx,
                      double* Y, int64_t ldy, int nrhs, cudaStream_t s0) {
    const int64_t nx = op == HLRC_OP_N ? M->ncols : M->nrows;
    for (int r0 = 0; r0 < nrhs; r0 += MR_RB) {
        const cudaStream_t s = s0;
        // side stages read the block of x staged below and add into Y; the
        // next block overwrites it only after the join
        SideFork side{M, ws, s0};
        const int nr = std::min(MR_RB, nrhs - r0);
        const int64_t tot = nx * MR_RB;
        k_rows_from_cols<<<unsigned((tot + 255) / 256), 256, 0, s>>>(X, ldx, nx, r0, nr, ws.mr_x);
        M->launches += 1;
        HLRC_AFTER_LAUNCH("rows_from_cols");
        int nl = 0;   // kernels launched below, counted at their launch sites
        auto vec = [&](int name) -> double* {
            return name == V_X ? ws.mr_x : (name == V_T ? ws.mr_t : ws.mr_t2);
        };
        auto omap = [&](int name) -> OutMap {
            if (name == V_Y) return OutMap{Y + int64_t(r0) * ldy, 1, ldy, nr};
            return OutMap{vec(name), MR_RB, 1, MR_RB};
        };
        const double* A = reinterpret_cast<const double*>(M->store);
        const std::vector<Stage>& stl = mr_stages(M, op);
        thread_local std::vector<int> order;
        for (const int oi : stage_order(M, stl, order)) {
            const Stage& st = stl[size_t(oi)];
            const cudaStream_t s = side.before(st);
            if (st.kind == 2) {
                const DevTTPass& tp = M->tt[size_t(st.idx)];
                const int add = tp.mode != OUT_SET;
                const double alpha = tp.mode == OUT_ADD ? 1.0 : alpha_in;   // plain adds pass coefficients down a tree
                const OutMap om = omap(tp.out);
                if (ws.profile) prof_begin(M, stage_name(M, 2, st.idx), tp.alg_bytes, s);
                constexpr int TW = DMMA_WARPS;
                if (M->precision == HLRC_PREC_F64) {
                    if (tp.nsegs[FMT_F64] > 0) {
                        k_ttform_dmma<TW><<<tp.nsegs[FMT_F64], TW * 32, 0, s>>>(
                            tp.segs[FMT_F64], static_cast<const TTChunk*>(tp.chunks), A, vec(tp.in), om, ws.mr_part,
                            alpha, add);
                        ++nl;
                    }
                } else if (M->precision == HLRC_PREC_BFP) {
                    float* fpart = reinterpret_cast<float*>(ws.mr_part);
                    if (tp.nmseg[FMT_I24] > 0) {
                        k_ttform_bfp<true><<<tp.nmseg[FMT_I24], TC_WARPS * 32, bq_smem_t(true), s>>>(
                            tp.mseg[FMT_I24], tp.mcol, M->store, vec(tp.in), om, fpart, alpha, add);
                        ++nl;
                    }
                    if (tp.nmseg[FMT_I16] > 0) {
                        k_ttform_bfp<false><<<tp.nmseg[FMT_I16], TC_WARPS * 32, bq_smem_t(false), s>>>(
                            tp.mseg[FMT_I16], tp.mcol, M->store, vec(tp.in), om, fpart, alpha, add);
                        ++nl;
                    }
                } else {
                    const int n32 = tp.nmseg[FMT_F32];
                    float* fpart = reinterpret_cast<float*>(ws.mr_part);
                    if (tp.nmseg[FMT_BF16] > 0) {
                        k_ttform_mr<FMT_BF16><<<n32 + tp.nmseg[FMT_BF16], TC_WARPS * 32,
                                               tc_smem_bytes(TC_STAGE_TT, TC_STAGES_TT), s>>>(
                            tp.mseg[FMT_F32], n32, tp.mseg[FMT_BF16], tp.mcol, M->store, vec(tp.in), om, fpart, alpha, add);
                        ++nl;
                    } else if (n32 + tp.nmseg[FMT_F16] > 0) {
                        k_ttform_mr<FMT_F16><<<n32 + tp.nmseg[FMT_F16], TC_WARPS * 32,
                                               tc_smem_bytes(TC_STAGE_TT, TC_STAGES_TT), s>>>(
                            tp.mseg[FMT_F32], n32, tp.mseg[FMT_F16], tp.mcol, M->store, vec(tp.in), om, fpart, alpha, add);
                        ++nl;
                    }
                }
                if (ws.profile) prof_end(M, s);
                if (tp.ngroups > 0) {
                    if (ws.profile)
                        prof_begin(M, "ttfinish", tp.npart * MR_RB * (M->precision == HLRC_PREC_F64 ? 8 : 4), s);
                    // first level: runs of slots into the scratch part of the partials
                    const OutMap pm{ws.mr_part, MR_RB, 1, MR_RB};
                    float* fpart = reinterpret_cast<float*>(ws.mr_part);
                    const int b1 = fin_gpb(tp.ngroups1), b2 = fin_gpb(tp.ngroups);
                    const unsigned fg1 = unsigned((tp.ngroups1 + b1 - 1) / b1);
                    const unsigned fg = unsigned((tp.ngroups + b2 - 1) / b2);
                    if (M->precision == HLRC_PREC_F64) {
                        if (tp.ngroups1 > 0)
                            k_ttfinish_flat<MR_RB, double, false><<<fg1, 256, 0, s>>>(
                                tp.groups1, tp.ngroups1, b1, ws.mr_part, pm, static_cast<double*>(nullptr), 1.0, 0);
                        k_ttfinish_flat<MR_RB, double, false><<<fg, 256, 0, s>>>(
                            tp.groups, tp.ngroups, b2, ws.mr_part, om, static_cast<double*>(nullptr), alpha, add);
                    } else {
                        if (tp.ngroups1 > 0)
                            k_ttfinish_flat<MR_RB, float, true><<<fg1, 256, 0, s>>>(tp.groups1, tp.ngroups1, b1, fpart,
                                                                                    pm, fpart, 1.0, 0);
                        k_ttfinish_flat<MR_RB, float, false><<<fg, 256, 0, s>>>(
                            tp.groups, tp.ngroups, b2, fpart, om, static_cast<float*>(nullptr), alpha, add);
                    }
                    nl += 1 + (tp.ngroups1 > 0 ? 1 : 0);
                    if (ws.profile) prof_end(M, s);
                }
                HLRC_AFTER_LAUNCH(stage_name(M, 2, st.idx));
            } else if (st.kind == 1) {
                const DevNPass& np = M->n[size_t(st.idx)];
                if (np.launches() == 0) continue;
                if (np.ncta > 0) return fail(HLRC_ERR_INTERNAL, "tree sweep in a multi-vector product");
                if (ws.profile) prof_begin(M, stage_name(M, 1, st.idx), np.alg_bytes, s);
                const int add = np.mode != OUT_SET;
                const double alpha = np.mode == OUT_ADD ? 1.0 : alpha_in;   // plain adds pass coefficients down a tree
                const OutMap om = omap(np.out);
                constexpr int NW = DMMA_WARPS;
                const bool f64plan = M->precision == HLRC_PREC_F64;
                // the formats of one output tile run as separate grids, each
                // adding its share to the output in a fixed launch order
                if (f64plan && np.nsegs[FMT_F64] > 0) {
                    k_nform_dmma<NW><<<np.nsegs[FMT_F64], NW * 32, 0, s>>>(
                        np.segs[FMT_F64], static_cast<const NChunk*>(np.chunks), A, vec(np.vx), vec(np.vt), om, alpha,
                        add);
                    ++nl;
                }
                if (!f64plan && np.nmseg[FMT_F32] > 0) {
                    k_nform_d32<<<np.nmseg[FMT_F32], TC_WARPS * 32, tc_smem_bytes(TC_STAGE_N32, TC_STAGES_D32), s>>>(
                        np.mseg[FMT_F32], np.mcol, M->store, vec(np.vx), vec(np.vt), om, alpha, add);
                    ++nl;
                }
                if (!f64plan && np.nmseg[FMT_F16] > 0) {
                    k_nform_tc<FMT_F16><<<np.nmseg[FMT_F16], TC_WARPS * 32,
                                          tc_smem_bytes(TC_STAGE_N16, TC_STAGES_N16), s>>>(
                        np.mseg[FMT_F16], np.mcol, M->store, vec(np.vx), vec(np.vt), om, alpha, add);
                    ++nl;
                }
                if (!f64plan && np.nmseg[FMT_BF16] > 0) {
                    k_nform_tc<FMT_BF16><<<np.nmseg[FMT_BF16], TC_WARPS * 32,
                                           tc_smem_bytes(TC_STAGE_N16, TC_STAGES_N16), s>>>(
                        np.mseg[FMT_BF16], np.mcol, M->store, vec(np.vx), vec(np.vt), om, alpha, add);
                    ++nl;
                }
                if (!f64plan && np.nmseg[FMT_I24] > 0) {
                    k_nform_bfp<true><<<np.nmseg[FMT_I24], TC_WARPS * 32, bq_smem_n(true), s>>>(
                        np.mseg[FMT_I24], np.mcol, M->store, vec(np.vx), vec(np.vt), om, alpha, add);
                    ++nl;
                }
                if (!f64plan && np.nmseg[FMT_I16] > 0) {
                    k_nform_bfp<false><<<np.nmseg[FMT_I16], TC_WARPS * 32, bq_smem_n(false), s>>>(
                        np.mseg[FMT_I16], np.mcol, M->store, vec(np.vx), vec(np.vt), om, alpha, add);
                    ++nl;
                }
                if (ws.profile) prof_end(M, s);
                HLRC_AFTER_LAUNCH(stage_name(M, 1, st.idx));
            }
        }
        M->launches += nl;
        if (const cudaError_t fe = side.end(); fe != cudaSuccess)
            return fail(HLRC_ERR_CUDA, "side stream: %s", cudaGetErrorString(fe));
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(HLRC_ERR_CUDA, "kernel launch failed: %s", cudaGetErrorString(e));
    return HLRC_OK;
}

// Can the product take the one-pass 64-vector kernels?  16-bit H stores,
// op N, a workspace with their arrays, and at least wide_min_nrhs vectors.
bool wide_ok(hlrc_hmat M, const Workspace& ws, int op, int nrhs) {
    return M->wide && op == HLRC_OP_N && ws.w_xs && nrhs >= M->wide_min_nrhs && nrhs >= 2;
}

// y := y + alpha M X for nrhs vectors, WIDE_RHS per pass: x is split into
// 16-bit terms once, the tile T-form writes t's split rows (multi-tile
// outputs through FP32 partials and the finish), and the N-form adds
// alpha (U t + D x) to Y.  The matrix is streamed once per 64 vectors.
hlrc_status run_wide(hlrc_hmat M, const Workspace& ws, double alpha, const double* X, int64_t ldx, double* Y,
                     int64_t ldy, int nrhs, cudaStream_t s) {
    const int f = wide_format(M);
    if (f < 0) return fail(HLRC_ERR_INTERNAL, "64-vector product on a handle without 64-vector passes");
    const std::vector<Stage>& st = M->stages[HLRC_OP_N];
    const DevTTPass& tp = M->tt[size_t(st[0].idx)];
    const DevNPass& np = M->n[size_t(st[1].idx)];
    const int64_t nx = M->ncols;
    const bool bf = f == FMT_BF16;
    for (int r0 = 0; r0 < nrhs; r0 += WIDE_RHS) {
        const int nr = std::min(WIDE_RHS, nrhs - r0);
        const double* Xr = X + int64_t(r0) * ldx;
        if (ws.profile) prof_begin(M, "wide_xsplit", nx * int64_t(nr) * 8 + nx * WIDE_ROWB, s);
        HLRC_CUDA(cudaMemsetAsync(ws.w_xmax, 0, WIDE_RHS * sizeof(unsigned long long), s));
        const unsigned gx = unsigned(std::min<int64_t>((nx + 255) / 256, 4 * 148));
        k_wide_xmax<<<dim3(std::max(1u, gx), unsigned(nr)), 256, 0, s>>>(Xr, ldx, nx, nr, ws.w_xmax);
        const unsigned gs = unsigned(std::max<int64_t>(1, (nx + TILE - 1) / TILE));
        if (bf) k_wide_xsplit<FMT_BF16><<<gs, 256, 0, s>>>(Xr, ldx, nx, nr, ws.w_xmax, ws.w_xs, ws.w_g);
        else k_wide_xsplit<FMT_F16><<<gs, 256, 0, s>>>(Xr, ldx, nx, nr, ws.w_xmax, ws.w_xs, ws.w_g);
        if (ws.profile) prof_end(M, s);
        M->launches += 2;
        HLRC_AFTER_LAUNCH("wide_xsplit");
        // full-tile units through TMA (persistent CTAs, two per SM), the
        // others through cp.async; the same outputs are never written by both
        const bool tma = M->tma && ws.has_tm;
        const int ntma = tma ? M->w_nunits_tma : 0;
        const WTUnit* ucp = tma ? M->w_units : M->w_units_tma;   // without TMA every unit takes cp.async
        const int ncp = tma ? M->w_nunits : M->w_nunits + M->w_nunits_tma;
        const WaitCfg wc{M->wait_ns, M->wait_skip};
        if (ntma + ncp > 0) {
            if (ws.profile) prof_begin(M, stage_name(M, 2, st[0].idx), tp.alg_bytes, s);
            if (ntma > 0) {
                const int grid = std::min(ntma, 2 * M->sms);
                if (bf)
                    k_ctform_wtma<FMT_BF16><<<grid, WTMA_THREADS_C, wtma_smem_c(), s>>>(
                        M->w_units_tma, ntma, M->w_blks, M->w_slabs, M->w_tiles, M->w_ctab, M->tm_s8, ws.tm_x64,
                        ws.w_ts, ws.w_part, M->dev_err, wc);
                else
                    k_ctform_wtma<FMT_F16><<<grid, WTMA_THREADS_C, wtma_smem_c(), s>>>(
                        M->w_units_tma, ntma, M->w_blks, M->w_slabs, M->w_tiles, M->w_ctab, M->tm_s8, ws.tm_x64,
                        ws.w_ts, ws.w_part, M->dev_err, wc);
                M->launches += 1;
            }
            if (ncp > 0) {
                if (bf)
                    k_ctform_wide<FMT_BF16><<<ncp, WIDE_THREADS, wide_smem_c(), s>>>(
                        ucp, M->w_blks, M->w_slabs, M->w_tiles, M->store, ws.w_xs, ws.w_ts, M->w_texp, ws.w_part,
                        M->dev_err, wc);
                else
                    k_ctform_wide<FMT_F16><<<ncp, WIDE_THREADS, wide_smem_c(), s>>>(
                        ucp, M->w_blks, M->w_slabs, M->w_tiles, M->store, ws.w_xs, ws.w_ts, M->w_texp, ws.w_part,
                        M->dev_err, wc);
                M->launches += 1;
            }
            if (ws.profile) prof_end(M, s);
            HLRC_AFTER_LAUNCH(stage_name(M, 2, st[0].idx));
        }
        if (M->w_ngroups > 0) {
            if (ws.profile) prof_begin(M, "ttfinish", M->w_npart * WIDE_RHS * 4, s);
            if (bf)
                k_ttfinish_wide<FMT_BF16><<<(M->w_ngroups + 7) / 8, 256, 0, s>>>(M->w_groups, M->w_ngroups, ws.w_part,
                                                                                  ws.w_ts, M->w_texp);
            else
                k_ttfinish_wide<FMT_F16><<<(M->w_ngroups + 7) / 8, 256, 0, s>>>(M->w_groups, M->w_ngroups, ws.w_part,
                                                                                 ws.w_ts, M->w_texp);
            if (ws.profile) prof_end(M, s);
            M->launches += 1;
            HLRC_AFTER_LAUNCH("ttfinish");
        }
        // full 64-row tiles through TMA, the other tiles (and everything,
        // when TMA is unavailable) through cp.async
        const int nwt = tma ? np.nwseg : 0;
        const MSeg* mcp = tma ? np.mseg_cp : np.mseg[f];
        const int nmcp = tma ? np.nmseg_cp : np.nmseg[f];
        if (nwt + nmcp > 0) {
            const OutMap om{Y + int64_t(r0) * ldy, 1, ldy, nr};
            if (ws.profile) prof_begin(M, stage_name(M, 1, st[1].idx), np.alg_bytes, s);
            if (nwt > 0) {
                if (bf)
                    k_nform_wtma<FMT_BF16><<<nwt, WTMA_THREADS, wtma_smem_n(), s>>>(
                        np.wseg, np.wstage, M->tm_s16, ws.tm_x16, ws.tm_t16, ws.w_g, om, alpha, M->dev_err, wc);
                else
                    k_nform_wtma<FMT_F16><<<nwt, WTMA_THREADS, wtma_smem_n(), s>>>(
                        np.wseg, np.wstage, M->tm_s16, ws.tm_x16, ws.tm_t16, ws.w_g, om, alpha, M->dev_err, wc);
                M->launches += 1;
            }
            if (nmcp > 0) {
                if (bf)
                    k_nform_wide<FMT_BF16><<<nmcp, WIDE_THREADS, wide_smem_n(), s>>>(
                        mcp, np.wcol, M->store, ws.w_xs, ws.w_ts, ws.w_g, om, alpha, 1, M->dev_err, wc);
                else
                    k_nform_wide<FMT_F16><<<nmcp, WIDE_THREADS, wide_smem_n(), s>>>(
                        mcp, np.wcol, M->store, ws.w_xs, ws.w_ts, ws.w_g, om, alpha, 1, M->dev_err, wc);
                M->launches += 1;
            }
            if (ws.profile) prof_end(M, s);
            HLRC_AFTER_LAUNCH(stage_name(M, 1, st[1].idx));
        }
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(HLRC_ERR_CUDA, "kernel launch failed: %s", cudaGetErrorString(e));
    return HLRC_OK;
}

hlrc_status check_mvm_args(hlrc_hmat M, int op, const double* x, double* y, int nrhs, int64_t ldx, int64_t ldy) {
    if (!M) return fail(HLRC_ERR_ARG, "matrix handle is NULL");
    if (op < 0 || op > 2) return fail(HLRC_ERR_ARG, "op %d is not a valid hlrc_op", op);
    if (M->stages[op].empty())
        return fail(HLRC_ERR_UNSUPPORTED_OP, "op %d is not supported for this matrix (uniform-H: N and C only)", op);
    if (nrhs < 0) return fail(HLRC_ERR_ARG, "nrhs < 0");
    const int64_t nx = op == HLRC_OP_N ? M->ncols : M->nrows;
    const int64_t ny = op == HLRC_OP_N ? M->nrows : M->ncols;
    if (nrhs > 1 && (ldx < nx || ldy < ny)) return fail(HLRC_ERR_SHAPE, "ldx/ldy smaller than the vector length");
    if (nrhs > 0 && ((nx > 0 && !x) || (ny > 0 && !y))) return fail(HLRC_ERR_ARG, "x or y is NULL");
    return HLRC_OK;
}

}  // namespace

extern "C" hlrc_status hlrc_upload_h(const hlrc_h_desc* desc, const hlrc_options* opts, hlrc_hmat* out) {
    clear_error();
    if (!desc || !out) return fail(HLRC_ERR_ARG, "hlrc_upload_h: null argument");
    *out = nullptr;
    hlrc_options o;
    if (opts) o = *opts; else hlrc_default_options(&o);
    Plan p;
    const hlrc_status st = plan_h_leaves(*desc, o, p);
    if (st != HLRC_OK) return st;
    return upload_plan(p, o, out);
}

extern "C" hlrc_status hlrc_upload_h_batch(const hlrc_h_desc* descs, int count, const int64_t* offsets,
                                           const hlrc_options* opts, hlrc_hmat* out) {
    clear_error();
    if (!descs || !offsets || !out || count < 1) return fail(HLRC_ERR_ARG, "hlrc_upload_h_batch: bad argument");
    *out = nullptr;
    hlrc_options o;
    if (opts) o = *opts; else hlrc_default_options(&o);
    std::vector<hlrc_block> all;
    double area = 0;
    for (int i = 0; i < count; ++i) {
        const hlrc_h_desc& d = descs[i];
        if (d.nrows != d.ncols) return fail(HLRC_ERR_SHAPE, "batch member %d is not square", i);
        if (offsets[i] < 0 || offsets[i] + d.nrows > offsets[i + 1])
            return fail(HLRC_ERR_SHAPE, "batch member %d does not fit between offsets %lld and %lld", i,
                        (long long)offsets[i], (long long)offsets[i + 1]);
        if (d.nblocks > 0 && !d.blocks) return fail(HLRC_ERR_ARG, "batch member %d: blocks == NULL", i);
        double a = 0;
        for (int64_t b = 0; b < d.nblocks; ++b) {
            hlrc_block blk = d.blocks[b];
            if (blk.row0 < 0 || blk.col0 < 0 || blk.nrows < 0 || blk.ncols < 0 || blk.row0 + blk.nrows > d.nrows ||
                blk.col0 + blk.ncols > d.ncols)
                return fail(HLRC_ERR_SHAPE, "batch member %d, block %lld: index set outside the member", i,
                            (long long)b);
            a += double(blk.nrows) * double(blk.ncols);
            blk.row0 += offsets[i];
            blk.col0 += offsets[i];
            all.push_back(blk);
        }
        if (a != double(d.nrows) * double(d.ncols))
            return fail(HLRC_ERR_SHAPE, "batch member %d: leaves cover %.0f of %.0f entries", i, a,
                        double(d.nrows) * double(d.ncols));
        area += a;
    }
    Plan p;
    const hlrc_h_desc cd{offsets[count], offsets[count], int64_t(all.size()), all.data()};
    const hlrc_status st = plan_h_leaves(cd, o, p, area);
    if (st != HLRC_OK) return st;
    return upload_plan(p, o, out);
}

extern "C" hlrc_status hlrc_upload_uniform(const hlrc_uniform_desc* desc, const hlrc_options* opts, hlrc_hmat* out) {
    clear_error();
    if (!desc || !out) return fail(HLRC_ERR_ARG, "hlrc_upload_uniform: null argument");
    *out = nullptr;
    hlrc_options o;
    if (opts) o = *opts; else hlrc_default_options(&o);
    Plan p;
    hlrc_status st = plan_uniform(*desc, o, p);
    if (st != HLRC_OK) return st;
    return upload_plan(p, o, out);
}

extern "C" hlrc_status hlrc_plan_info_h(const hlrc_h_desc* desc, const hlrc_options* opts, hlrc_info* info) {
    clear_error();
    if (!desc || !info) return fail(HLRC_ERR_ARG, "hlrc_plan_info_h: null argument");
    hlrc_options o;
    if (opts) o = *opts; else hlrc_default_options(&o);
    Plan p;
    hlrc_status st = plan_h_leaves(*desc, o, p);
    if (st != HLRC_OK) return st;
    if (st = check_streams(p); st != HLRC_OK) return st;
    fill_info(p, arena_layout(p), *info);
    return HLRC_OK;
}

extern "C" hlrc_status hlrc_upload_h2(const hlrc_h2_desc* desc, const hlrc_options* opts, hlrc_hmat* out) {
    clear_error();
    if (!desc || !out) return fail(HLRC_ERR_ARG, "hlrc_upload_h2: null argument");
    *out = nullptr;
    hlrc_options o;
    if (opts) o = *opts; else hlrc_default_options(&o);
    Plan p;
    hlrc_status st = plan_h2(*desc, o, p);
    if (st != HLRC_OK) return st;
    return upload_plan(p, o, out);
}

extern "C" hlrc_status hlrc_plan_info_h2(const hlrc_h2_desc* desc, const hlrc_options* opts, hlrc_info* info) {
    clear_error();
    if (!desc || !info) return fail(HLRC_ERR_ARG, "hlrc_plan_info_h2: null argument");
    hlrc_options o;
    if (opts) o = *opts; else hlrc_default_options(&o);
    Plan p;
    hlrc_status st = plan_h2(*desc, o, p);
    if (st != HLRC_OK) return st;
    if (st = check_streams(p); st != HLRC_OK) return st;
    fill_info(p, arena_layout(p), *info);
    return HLRC_OK;
}

extern "C" hlrc_status hlrc_plan_info_uniform(const hlrc_uniform_desc* desc, const hlrc_options* opts,
                                              hlrc_info* info) {
    clear_error();
    if (!desc || !info) return fail(HLRC_ERR_ARG, "hlrc_plan_info_uniform: null argument");
    hlrc_options o;
    if (opts) o = *opts; else hlrc_default_options(&o);
    Plan p;
    hlrc_status st = plan_uniform(*desc, o, p);
    if (st != HLRC_OK) return st;
    if (st = check_streams(p); st != HLRC_OK) return st;
    fill_info(p, arena_layout(p), *info);
    return HLRC_OK;
}

extern "C" hlrc_status hlrc_mvm(hlrc_hmat M, double alpha, int op, const double* x, double* y, int nrhs,
                                int64_t ldx, int64_t ldy, void* stream) {
    clear_error();
    hlrc_status st = check_mvm_args(M, op, x, y, nrhs, ldx, ldy);
    if (st != HLRC_OK) return st;
    if (alpha == 0.0 || nrhs == 0) return HLRC_OK;
    DeviceGuard g(M->device);
    if (!g.ok) return fail(HLRC_ERR_CUDA, "cannot select device %d", M->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const Workspace ws = handle_workspace(M);
    if (wide_ok(M, ws, op, nrhs)) return run_wide(M, ws, alpha, x, ldx, y, ldy, nrhs, s);
    if (multi_rhs_ok(M, ws, op, nrhs)) return run_multi(M, ws, alpha, op, x, ldx, y, ldy, nrhs, s);
    for (int r = 0; r < nrhs; ++r) {
        st = run_single(M, ws, alpha, op, x + size_t(r) * size_t(ldx), y + size_t(r) * size_t(ldy), s);
        if (st != HLRC_OK) return st;
    }
    return HLRC_OK;
}

extern "C" hlrc_status hlrc_mvm_host(hlrc_hmat M, double alpha, int op, const double* x, double* y, int nrhs,
                                     int64_t ldx, int64_t ldy) {
    clear_error();
    hlrc_status st = check_mvm_args(M, op, x, y, nrhs, ldx, ldy);
    if (st != HLRC_OK) return st;
    if (alpha == 0.0 || nrhs == 0) return HLRC_OK;
    DeviceGuard g(M->device);
    if (!g.ok) return fail(HLRC_ERR_CUDA, "cannot select device %d", M->device);
    const int64_t nx = op == HLRC_OP_N ? M->ncols : M->nrows;
    const int64_t ny = op == HLRC_OP_N ? M->nrows : M->ncols;
    const size_t ex = size_t(nx) * size_t(nrhs), ey = size_t(ny) * size_t(nrhs);
    // the staging buffers and the handle's workspace serve one host call at a time
    std::lock_guard<std::mutex> lock(M->host_mu);
    if (ex > M->hx_elems) {
        cudaFree(M->hx);
        M->hx = nullptr;
        HLRC_CUDA(cudaMalloc(&M->hx, std::max<size_t>(ex, 1) * sizeof(double)));
        M->hx_elems = ex;
    }
    if (ey > M->hy_elems) {
        cudaFree(M->hy);
        M->hy = nullptr;
        HLRC_CUDA(cudaMalloc(&M->hy, std::max<size_t>(ey, 1) * sizeof(double)));
        M->hy_elems = ey;
    }
    const int64_t lx = nrhs > 1 ? ldx : nx, ly = nrhs > 1 ? ldy : ny;
    HLRC_CUDA(cudaMemcpy2D(M->hx, size_t(nx) * 8, x, size_t(lx) * 8, size_t(nx) * 8, size_t(nrhs), cudaMemcpyHostToDevice));
    HLRC_CUDA(cudaMemcpy2D(M->hy, size_t(ny) * 8, y, size_t(ly) * 8, size_t(ny) * 8, size_t(nrhs), cudaMemcpyHostToDevice));
    const Workspace ws = handle_workspace(M);
    if (wide_ok(M, ws, op, nrhs)) {
        st = run_wide(M, ws, alpha, M->hx, nx, M->hy, ny, nrhs, nullptr);
        if (st != HLRC_OK) return st;
    } else if (multi_rhs_ok(M, ws, op, nrhs)) {
        st = run_multi(M, ws, alpha, op, M->hx, nx, M->hy, ny, nrhs, nullptr);
        if (st != HLRC_OK) return st;
    } else {
        for (int r = 0; r < nrhs; ++r) {
            st = run_single(M, ws, alpha, op, M->hx + size_t(r) * size_t(nx), M->hy + size_t(r) * size_t(ny), nullptr);
            if (st != HLRC_OK) return st;
        }
    }
    HLRC_CUDA(cudaMemcpy2D(y, size_t(ly) * 8, M->hy, size_t(ny) * 8, size_t(ny) * 8, size_t(nrhs), cudaMemcpyDeviceToHost));
    return HLRC_OK;
}

extern "C" hlrc_status hlrc_get_info(hlrc_hmat M, hlrc_info* info) {
    if (!M || !info) return fail(HLRC_ERR_ARG, "hlrc_get_info: null argument");
    *info = M->info;
    return HLRC_OK;
}

extern "C" hlrc_status hlrc_get_tuning(hlrc_hmat M, hlrc_tuning* t) {
    if (!M || !t) return fail(HLRC_ERR_ARG, "hlrc_get_tuning: null argument");
    std::memset(t, 0, sizeof(*t));
    t->nform_warps = M->nform_warps;
    t->ttform_warps = M->ttform_warps;
    t->mr_min_nrhs = M->mr_min_nrhs;
    t->wide_min_nrhs = M->wide_min_nrhs;
    t->overlap = M->overlap;
    t->side_at = M->side_at;
    return HLRC_OK;
}

extern "C" hlrc_status hlrc_set_tuning(hlrc_hmat M, const hlrc_tuning* t) {
    if (!M || !t) return fail(HLRC_ERR_ARG, "hlrc_set_tuning: null argument");
    auto warps_ok = [](int w) { return w == 4 || w == 8 || w == 16; };
    if (!warps_ok(t->nform_warps) || !warps_ok(t->ttform_warps))
        return fail(HLRC_ERR_ARG, "hlrc_set_tuning: warps per CTA must be 4, 8 or 16 (got %d, %d)", t->nform_warps,
                    t->ttform_warps);
    if (t->mr_min_nrhs < 2 || t->mr_min_nrhs > HLRC_MR_NEVER)
        return fail(HLRC_ERR_ARG, "hlrc_set_tuning: mr_min_nrhs must be in [2, %d] (got %d)", HLRC_MR_NEVER,
                    t->mr_min_nrhs);
    if (t->wide_min_nrhs < 2 || t->wide_min_nrhs > HLRC_MR_NEVER)
        return fail(HLRC_ERR_ARG, "hlrc_set_tuning: wide_min_nrhs must be in [2, %d] (got %d)", HLRC_MR_NEVER,
                    t->wide_min_nrhs);
    if (t->overlap != 0 && t->overlap != 1)
        return fail(HLRC_ERR_ARG, "hlrc_set_tuning: overlap must be 0 or 1 (got %d)", t->overlap);
    if (t->side_at < 0 || t->side_at > 16)
        return fail(HLRC_ERR_ARG, "hlrc_set_tuning: side_at must be in [0, 16] (got %d)", t->side_at);
    // every field is checked before any is set
    M->nform_warps = t->nform_warps;
    M->ttform_warps = t->ttform_warps;
    M->mr_min_nrhs = t->mr_min_nrhs;
    M->wide_min_nrhs = t->wide_min_nrhs;
    M->overlap = t->overlap;
    M->side_at = t->side_at;
    return HLRC_OK;
}

extern "C" hlrc_status hlrc_set_profiling(hlrc_hmat M, int enable) {
    if (!M) return fail(HLRC_ERR_ARG, "hlrc_set_profiling: null handle");
    M->profiling = enable != 0;
    M->nprof = 0;
    return HLRC_OK;
}

extern "C" int hlrc_last_profile(hlrc_hmat M, const char** names, int* count, double* ms, int64_t* bytes,
                                 int cap) {
    if (!M) return 0;
    int n = 0;
    for (int i = 0; i < M->nprof; ++i) {
        const ProfileRec& r = M->prof[size_t(i)];
        float t = 0.f;
        cudaEventSynchronize(r.e1);
        cudaEventElapsedTime(&t, r.e0, r.e1);
        int k = 0;
        while (k < n && names && std::strcmp(names[k], r.name) != 0) ++k;
        if (k == n) {
            if (n >= cap) continue;
            if (names) names[n] = r.name;
            if (count) count[n] = 0;
            if (ms) ms[n] = 0.0;
            if (bytes) bytes[n] = r.alg_bytes;
            ++n;
        }
        if (count) count[k] += 1;
        if (ms) ms[k] += double(t);
    }
    M->nprof = 0;
    return n;
}

extern "C" hlrc_status hlrc_debug_waits(hlrc_hmat M, int64_t limit_ns, int skip_handover) {
    clear_error();
    if (!M) return fail(HLRC_ERR_ARG, "hlrc_debug_waits: null handle");
    if (limit_ns < 0 || limit_ns > int64_t(60) * 1000000000) return fail(HLRC_ERR_ARG, "hlrc_debug_waits: limit out of range");
    M->wait_ns = limit_ns > 0 ? uint64_t(limit_ns) : 2000000000ull;
    M->wait_skip = skip_handover != 0;
    return HLRC_OK;
}

extern "C" hlrc_status hlrc_check_device_error(hlrc_hmat M, int* code) {
    clear_error();
    if (!M || !code) return fail(HLRC_ERR_ARG, "hlrc_check_device_error: null argument");
    *code = 0;
    DeviceGuard g(M->device);
    if (!g.ok) return fail(HLRC_ERR_CUDA, "cannot select device %d", M->device);
    HLRC_CUDA(cudaMemcpy(code, M->dev_err, sizeof(int), cudaMemcpyDeviceToHost));
    HLRC_CUDA(cudaMemset(M->dev_err, 0, sizeof(int)));
    return HLRC_OK;
}

// ------------------------------------------------------------------------
// hlrc_mvm_noalloc: the product with its scratch in a static device array.
//
// The scratch of one product (low-rank coefficients t, the second
// coefficient array of uniform-H, and the per-tile partial sums) lives in
// this file-scope array instead of the handle's workspace.  Each device that
// loads the library holds its own 8 MiB copy until the process exits.
// Host code must not use `g_noalloc_scratch` as a pointer (on the host it
// names a stand-in, not device memory): its device address is obtained once
// per device with cudaGetSymbolAddress while that device is current.
constexpr size_t NOALLOC_SCRATCH_DOUBLES = size_t(1) << 20;  // 8 MiB
static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_SCRATCH_DOUBLES];

namespace {
constexpr int NOALLOC_MAX_DEVICES = 128;
std::mutex g_noalloc_mu;
double* g_noalloc_ptr[NOALLOC_MAX_DEVICES] = {};

// device address of the scratch on `dev` (which must be current)
hlrc_status noalloc_scratch(int dev, double** out) {
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES)
        return fail(HLRC_ERR_ARG, "hlrc_mvm_noalloc: device ordinal %d outside 0..%d", dev, NOALLOC_MAX_DEVICES - 1);
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess)
            return fail(HLRC_ERR_CUDA, "hlrc_mvm_noalloc: cudaGetSymbolAddress on device %d failed: %s", dev,
                        cudaGetErrorString(e));
        g_noalloc_ptr[dev] = static_cast<double*>(p);
    }
    *out = g_noalloc_ptr[dev];
    return HLRC_OK;
}
}  // namespace

extern "C" hlrc_status hlrc_mvm_noalloc(hlrc_hmat M, double alpha, int op, const double* x, double* y,
                                        void* stream) {
    clear_error();
    hlrc_status st = check_mvm_args(M, op, x, y, 1, 0, 0);
    if (st != HLRC_OK) return st;
    if (alpha == 0.0) return HLRC_OK;
    const size_t need = size_t(std::max<int64_t>(1, M->n_t)) + size_t(std::max<int64_t>(1, M->n_t2)) +
                        size_t(M->n_part);
    if (need > NOALLOC_SCRATCH_DOUBLES)
        return fail(HLRC_ERR_SHAPE,
                    "hlrc_mvm_noalloc: this matrix needs %zu doubles (%.1f MiB) of scratch, the static scratch "
                    "holds %zu doubles (8 MiB); use hlrc_mvm",
                    need, double(need) * 8.0 / 1048576.0, NOALLOC_SCRATCH_DOUBLES);
    DeviceGuard g(M->device);
    if (!g.ok) return fail(HLRC_ERR_CUDA, "cannot select device %d", M->device);
    double* base = nullptr;
    st = noalloc_scratch(M->device, &base);
    if (st != HLRC_OK) return st;
    // every scratch entry a product reads is written earlier in the same
    // product (coefficients with OUT_SET, each partial by its chunk), so the
    // previous call's contents need no clearing
    Workspace ws;
    ws.t = base;
    ws.t2 = base + std::max<int64_t>(1, M->n_t);
    ws.part = base + std::max<int64_t>(1, M->n_t) + std::max<int64_t>(1, M->n_t2);
    return run_single(M, ws, alpha, op, x, y, static_cast<cudaStream_t>(stream));
}

extern "C" int64_t hlrc_launch_count(hlrc_hmat M) { return M ? M->launches.load() : 0; }

// ------------------------------------------------------------------------
// Workspaces: scratch owned by the caller, one per concurrent stream.
//
// A handle is immutable after upload; everything a product writes besides y
// is scratch.  HLR's TBB product may run concurrently on one matrix with
// different y (tbb/arith.hh:312-323, y locked per 64-row chunk in
// tbb/detail/arith.hh:95-124); here the same is had by giving each stream
// its own workspace.
struct hlrc_workspace_s {
    int device = 0;
    int64_t n_t = 0, n_t2 = 0, n_part = 0;   // one-vector capacities (doubles)
    size_t mr_nx = 0, mr_nt = 0, mr_nt2 = 0, mr_np = 0;   // multi-vector capacities (0: none)
    size_t w_xs = 0, w_ts = 0, w_part = 0;                // 64-vector capacities in bytes (0: none)
    char* arena = nullptr;
    size_t bytes = 0;
    Workspace ws;
};

extern "C" hlrc_status hlrc_workspace_create(hlrc_hmat M, int max_nrhs, hlrc_workspace* out) {
    clear_error();
    if (!M || !out) return fail(HLRC_ERR_ARG, "hlrc_workspace_create: null argument");
    *out = nullptr;
    if (max_nrhs < 1) return fail(HLRC_ERR_ARG, "hlrc_workspace_create: max_nrhs %d < 1", max_nrhs);
    DeviceGuard g(M->device);
    if (!g.ok) return fail(HLRC_ERR_CUDA, "cannot select device %d", M->device);
    auto W = std::make_unique<hlrc_workspace_s>();
    W->device = M->device;
    W->n_t = std::max<int64_t>(1, M->n_t);
    W->n_t2 = std::max<int64_t>(1, M->n_t2);
    W->n_part = std::max<int64_t>(1, M->n_part);
    size_t off = 0;
    auto take = [&](size_t elems) { const size_t o_ = off; off = align_up(off + elems * sizeof(double), 256); return o_; };
    const size_t o_t = take(size_t(W->n_t)), o_t2 = take(size_t(W->n_t2)), o_p = take(size_t(W->n_part));
    MrSizes z;
    size_t o_mr = 0;
    if (max_nrhs > 1 && has_multi_kernels(M)) {
        z = mr_sizes(M);
        o_mr = take(z.bytes / sizeof(double) + 1);
        W->mr_nx = z.nx; W->mr_nt = z.nt; W->mr_nt2 = z.nt2; W->mr_np = z.np;
    }
    WideSizes zw;
    size_t o_w = 0;
    if (max_nrhs > MR_RB && M->wide) {
        const hlrc_status st = enable_wide_smem(M->device);
        if (st != HLRC_OK) return st;
        zw = wide_sizes(M);
        o_w = take(zw.bytes / sizeof(double) + 1);
        W->w_xs = zw.xs; W->w_ts = zw.ts; W->w_part = zw.part;
    }
    W->bytes = off;
    const cudaError_t e = cudaMalloc(&W->arena, W->bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(HLRC_ERR_OOM, "hlrc_workspace_create: cudaMalloc of %zu bytes failed: %s", W->bytes,
                    cudaGetErrorString(e));
    }
    W->ws.t = reinterpret_cast<double*>(W->arena + o_t);
    W->ws.t2 = reinterpret_cast<double*>(W->arena + o_t2);
    W->ws.part = reinterpret_cast<double*>(W->arena + o_p);
    if (W->mr_nx) z.carve(W->arena + o_mr, W->ws.mr_x, W->ws.mr_t, W->ws.mr_t2, W->ws.mr_part);
    if (W->w_xs) {
        zw.carve(W->arena + o_w, W->ws);
        wide_ws_maps(M, W->ws);
    }
    W->ws.profile = false;
    if (has_side(M->stages_nf)) {
        if (const hlrc_status ss = side_create(W->ws); ss != HLRC_OK) {
            side_destroy(W->ws);
            cudaFree(W->arena);
            return ss;
        }
    }
    *out = W.release();
    return HLRC_OK;
}

extern "C" hlrc_status hlrc_workspace_free(hlrc_workspace W) {
    if (!W) return HLRC_OK;
    DeviceGuard g(W->device);
    cudaFree(W->arena);
    side_destroy(W->ws);
    delete W;
    return HLRC_OK;
}

extern "C" hlrc_status hlrc_mvm_ws(hlrc_hmat M, hlrc_workspace W, double alpha, int op, const double* x, double* y,
                                   int nrhs, int64_t ldx, int64_t ldy, void* stream) {
    clear_error();
    hlrc_status st = check_mvm_args(M, op, x, y, nrhs, ldx, ldy);
    if (st != HLRC_OK) return st;
    if (!W) return fail(HLRC_ERR_ARG, "hlrc_mvm_ws: workspace is NULL");
    if (W->device != M->device)
        return fail(HLRC_ERR_ARG, "hlrc_mvm_ws: workspace on device %d, matrix on device %d", W->device, M->device);
    if (W->n_t < M->n_t || W->n_t2 < M->n_t2 || W->n_part < M->n_part)
        return fail(HLRC_ERR_SHAPE, "hlrc_mvm_ws: workspace too small for this matrix (create it for this handle)");
    if (alpha == 0.0 || nrhs == 0) return HLRC_OK;
    DeviceGuard g(M->device);
    if (!g.ok) return fail(HLRC_ERR_CUDA, "cannot select device %d", M->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Workspace ws = W->ws;
    if (ws.mr_x) {   // the multi-vector arrays serve only handles they fit
        const MrSizes z = mr_sizes(M);
        if (!has_multi_kernels(M) || z.nx > W->mr_nx || z.nt > W->mr_nt || z.nt2 > W->mr_nt2 || z.np > W->mr_np)
            ws.mr_x = nullptr;
    }
    if (ws.w_xs) {
        const WideSizes z = wide_sizes(M);
        if (!M->wide || z.xs > W->w_xs || z.ts > W->w_ts || z.part > W->w_part) ws.w_xs = nullptr;
    }
    if (wide_ok(M, ws, op, nrhs)) return run_wide(M, ws, alpha, x, ldx, y, ldy, nrhs, s);
    if (multi_rhs_ok(M, ws, op, nrhs)) return run_multi(M, ws, alpha, op, x, ldx, y, ldy, nrhs, s);
    for (int r = 0; r < nrhs; ++r) {
        st = run_single(M, ws, alpha, op, x + size_t(r) * size_t(ldx), y + size_t(r) * size_t(ldy), s);
        if (st != HLRC_OK) return st;
    }
    return HLRC_OK;
}

extern "C" hlrc_status hlrc_free(hlrc_hmat M) {
    if (!M) return HLRC_OK;
    DeviceGuard g(M->device);
    for (auto& r : M->prof) {
        cudaEventDestroy(r.e0);
        cudaEventDestroy(r.e1);
    }
    cudaFree(M->hx);
    cudaFree(M->hy);
    cudaFree(M->mr_arena);
    cudaFree(M->mr_tables);
    cudaFree(M->w_arena);
    cudaFree(M->w_static);
    cudaFree(M->arena);
    side_destroy(M->side_ws);
    delete M;
    return HLRC_OK;
}
