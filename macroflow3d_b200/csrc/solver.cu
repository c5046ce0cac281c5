// solver.cu -- host orchestration behind the C-ABI in include/mf3d.h.
//
// HeadSolver replaces the reference's FlowWorkspace + solve_head (src/physics/flow/
// solve_head.cu:75-243) for the PCG_MG path:
//   set_K : coarsen K to every level, build face coefficients (FP64 for the fine operator and
//           the coarse tail, FP32 / BF16 for a mixed-precision V-cycle), RHS, initial guess;
//   solve : r0 = b - A x0, then the PCG loop as ONE CUDA graph whose `while` node body is
//           [V-cycle -> z, <r,z>] [p = z + beta p] [Ap, <p,Ap>] [x, r update, stop test];
//           the stop test sets the while condition on the device, so the host waits once.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/mf3d.h"
#include "kernels_coarse.cuh"
#include "kernels_kfield.cuh"
#include "kernels_mg.cuh"
#include "kernels_nn.cuh"
#include "kernels_pcg.cuh"
#include "kernels_resid.cuh"
#include "kernels_setup.cuh"
#include "kernels_sweep_pair.cuh"
#include "kernels_sweep_tma.cuh"
#include "kernels_tail.cuh"
#include "kernels_velocity.cuh"

namespace mf3d {

static thread_local std::string g_err;

// Shared memory of the one-CTA coarse tail (padded x and b of its levels), at most.
static constexpr size_t kTailSmemMax = 200 * 1024;
// ... and of one CTA of the cluster kernel (x, b and the weights of its slabs)
static constexpr size_t kCoarseSmemMax = 224 * 1024;

// Device-time limit of one solve by default: the PCG loop stops with status 3 after this long
// (mf3d_head_solver_set_time_budget changes it per solver).
static constexpr unsigned long long kSolveBudgetNs = 120ull * 1000000000ull;

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define MF3D_CK(call)                                                                                   \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess)                                                                          \
            throw Error(e_ == cudaErrorMemoryAllocation ? MF3D_E_NOMEM : MF3D_E_CUDA,                   \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                            \
    } while (0)
// every kernel launch goes through this check; the counter feeds the launch statistics
static thread_local long long g_launches = 0;
#define MF3D_LAUNCH_CK()                                                                                \
    do {                                                                                                \
        ++g_launches;                                                                                   \
        MF3D_CK(cudaGetLastError());                                                                    \
    } while (0)

static int g_num_sms = 0;
static int num_sms() {
    if (g_num_sms == 0) {
        int dev = 0;
        MF3D_CK(cudaGetDevice(&dev));
        MF3D_CK(cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev));
    }
    return g_num_sms;
}

static unsigned grid1d(size_t n, int nt, int per_sm = 8) {
    const size_t want = (n + nt - 1) / nt;
    const size_t cap = (size_t)num_sms() * per_sm;
    return (unsigned)std::max<size_t>(1, std::min(want, cap));
}

// 3-D launch of the column-marching cell kernels: 32 x 8 threads per (x, y) tile, about
// per_sm * SMs blocks in total, each thread marching zchunk planes.
struct ColLaunch {
    dim3 grid, block;
    int zchunk;
    unsigned nblocks;
};
static ColLaunch col_launch(int nx, int ny, int nz, int per_sm = 8) {
    ColLaunch L;
    const long long gx = (nx + 31) / 32, gy = (ny + 7) / 8, bxy = gx * gy;
    long long nzc = std::max<long long>(1, std::min<long long>(nz, (long long)num_sms() * per_sm / std::max(1LL, bxy)));
    L.zchunk = (int)((nz + nzc - 1) / nzc);
    nzc = (nz + L.zchunk - 1) / L.zchunk;
    L.grid = dim3((unsigned)gx, (unsigned)gy, (unsigned)nzc);
    L.block = dim3(32, 8, 1);
    L.nblocks = (unsigned)(bxy * nzc);
    return L;
}

// RAII device allocation
struct DevMem {
    void* p = nullptr;
    size_t bytes = 0;
    DevMem() = default;
    explicit DevMem(size_t b) { alloc(b); }
    void alloc(size_t b) {
        release();
        bytes = b;
        if (b) MF3D_CK(cudaMalloc(&p, b));
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    ~DevMem() { release(); }
    DevMem(const DevMem&) = delete;
    DevMem& operator=(const DevMem&) = delete;
    template <class T> T* as() const { return static_cast<T*>(p); }
};

static BcDev to_dev(const mf3d_bc& bc) {
    BcDev d;
    for (int f = 0; f < 6; ++f) {
        d.type[f] = bc.type[f];
        d.value[f] = bc.value[f];
    }
    return d;
}

static void validate_bc(const mf3d_bc& bc) {
    // BCSpec::validate, src/core/BCSpec.hpp:66-86
    for (int a = 0; a < 3; ++a) {
        const bool p0 = bc.type[2 * a] == MF3D_BC_PERIODIC, p1 = bc.type[2 * a + 1] == MF3D_BC_PERIODIC;
        if (p0 != p1) throw Error(MF3D_E_INVALID, "Periodic BC must be specified on both faces of an axis");
    }
    for (int f = 0; f < 6; ++f) {
        if (bc.type[f] < 0 || bc.type[f] > 2) throw Error(MF3D_E_INVALID, "unknown BC type");
        if (!std::isfinite(bc.value[f])) throw Error(MF3D_E_INVALID, "BC values must be finite");
    }
}

static bool has_dirichlet(const mf3d_bc& bc) {
    for (int f = 0; f < 6; ++f)
        if (bc.type[f] == MF3D_BC_DIRICHLET) return true;
    return false;
}

// pin_enabled, src/numerics/pin_spec.hpp:109-120
static bool pin_enabled(int mode, const mf3d_bc& bc) {
    if (mode == MF3D_PIN_ON) return true;
    if (mode == MF3D_PIN_OFF) return false;
    return !has_dirichlet(bc);
}

struct Geom {
    int nx, ny, nz;
    size_t n;
    double dx;
};

// Work items of the x-pair sweep: (tile, z chunk) pairs, tiles fastest, about
// sp_items_per_cta() items per resident CTA; the grid is at most the resident CTA count and its
// CTAs walk the items in turn.  MF3D_SWEEP_ITEMS overrides the items per CTA (tuning).
static int sp_items_per_cta() {
    static int v = -1;
    if (v < 0) {
        const char* e = std::getenv("MF3D_SWEEP_ITEMS");
        v = e ? std::max(1, std::atoi(e)) : 1;
    }
    return v;
}
static dim3 pair_grid(const Geom& g, long long resident, int* zchunk, int tx = SP_TX) {
    const long long tiles = (long long)((g.nx + tx - 1) / tx) * ((g.ny + SP_TY - 1) / SP_TY);
    const long long want = resident * sp_items_per_cta();
    const long long nchunk = std::max<long long>(1, std::min<long long>(g.nz, want / std::max(1LL, tiles)));
    const int zc = (int)((g.nz + nchunk - 1) / nchunk);
    const long long items = tiles * ((g.nz + zc - 1) / zc);
    *zchunk = zc;
    return dim3((unsigned)std::max(1LL, std::min(items, resident)));
}

template <class T, class TC, bool TM>
static void launch_pair_sweep_tm(cudaStream_t s, dim3 grid, int mode, const SpMaps& m, const SpArgs<T, TC>& a) {
    const size_t smem = sp_smem_bytes<T, TC, TM>();
    switch (mode) {
    case 0: sweep_pair_kernel<T, TC, 0, TM><<<grid, SP_NT, smem, s>>>(m, a); break;
    case M_ZERO: sweep_pair_kernel<T, TC, M_ZERO, TM><<<grid, SP_NT, smem, s>>>(m, a); break;
    case M_PROLONG: sweep_pair_kernel<T, TC, M_PROLONG, TM><<<grid, SP_NT, smem, s>>>(m, a); break;
    case M_ZERO | M_PROLONG: sweep_pair_kernel<T, TC, M_ZERO | M_PROLONG, TM><<<grid, SP_NT, smem, s>>>(m, a); break;
    case M_DOT: sweep_pair_kernel<T, TC, M_DOT, TM><<<grid, SP_NT, smem, s>>>(m, a); break;
    case M_ZERO | M_DOT: sweep_pair_kernel<T, TC, M_ZERO | M_DOT, TM><<<grid, SP_NT, smem, s>>>(m, a); break;
    case M_PROLONG | M_DOT: sweep_pair_kernel<T, TC, M_PROLONG | M_DOT, TM><<<grid, SP_NT, smem, s>>>(m, a); break;
    case M_ZERO | M_PROLONG | M_DOT:
        sweep_pair_kernel<T, TC, M_ZERO | M_PROLONG | M_DOT, TM><<<grid, SP_NT, smem, s>>>(m, a);
        break;
    default: throw Error(MF3D_E_INVALID, "unsupported x-pair sweep mode");
    }
    MF3D_LAUNCH_CK();
}
template <class T, class TC>
static void launch_pair_sweep(cudaStream_t s, dim3 grid, int mode, bool tm, const SpMaps& m, const SpArgs<T, TC>& a) {
    if constexpr (!std::is_same<T, TC>::value) { // BF16 coefficients: TMA staging only
        if (!tm) throw Error(MF3D_E_INVALID, "x-pair sweep with BF16 coefficients needs TMA staging");
        launch_pair_sweep_tm<T, TC, true>(s, grid, mode, m, a);
    } else {
        if (tm) launch_pair_sweep_tm<T, TC, true>(s, grid, mode, m, a);
        else launch_pair_sweep_tm<T, TC, false>(s, grid, mode, m, a);
    }
}
// dynamic shared memory and resident CTAs per SM of one x-pair sweep variant
template <class T, class TC, int MODE, bool TM> static int pair_sweep_setup() {
    const size_t smem = sp_smem_bytes<T, TC, TM>();
    MF3D_CK(cudaFuncSetAttribute(sweep_pair_kernel<T, TC, MODE, TM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
    MF3D_CK(cudaFuncSetAttribute(sweep_pair_kernel<T, TC, MODE, TM>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 (int)cudaSharedmemCarveoutMaxShared));
    int n = 0;
    MF3D_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, sweep_pair_kernel<T, TC, MODE, TM>, SP_NT, smem));
    if (n < 1) throw Error(MF3D_E_CUDA, "x-pair sweep does not fit on an SM");
    return n;
}


// Levels by halving every axis (MGHierarchy, src/multigrid/mg_types.hpp:86-99): at most
// `max_levels`, stop when a coarse axis would be < 2.  An axis of odd length is never
// halved (the reference's 2:1 restriction is undefined there), so coarsening also stops
// at the first odd axis.
static std::vector<Geom> make_levels(const mf3d_grid& g, int max_levels) {
    std::vector<Geom> L;
    Geom c{g.nx, g.ny, g.nz, (size_t)g.nx * g.ny * g.nz, g.dx};
    for (int l = 0; l < std::max(1, max_levels); ++l) {
        L.push_back(c);
        if (l == max_levels - 1) break;
        if ((c.nx & 1) || (c.ny & 1) || (c.nz & 1)) break;
        Geom d{c.nx / 2, c.ny / 2, c.nz / 2, 0, c.dx * 2.0};
        if (d.nx < 2 || d.ny < 2 || d.nz < 2) break;
        d.n = (size_t)d.nx * d.ny * d.nz;
        c = d;
    }
    return L;
}

template <class TC> static LevelOp<TC> make_op(const Geom& G, const mf3d_bc& bc, bool pin, double scale) {
    LevelOp<TC> L{};
    L.nx = G.nx;
    L.ny = G.ny;
    L.nz = G.nz;
    L.per_x = bc.type[0] == MF3D_BC_PERIODIC;
    L.per_y = bc.type[2] == MF3D_BC_PERIODIC;
    L.per_z = bc.type[4] == MF3D_BC_PERIODIC;
    L.pin = pin ? 1 : 0;
    L.dx2 = G.dx * G.dx / scale;
    L.inv_dx2 = scale / (G.dx * G.dx);
    return L;
}

// Coefficient storage of one level in precision TC.
struct CoefStore {
    DevMem mem;
    template <class TC> void build(const Geom& G, size_t elt, LevelOp<TC>& L) {
        // every array starts on a 256-byte boundary (TMA needs 16)
        auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
        const size_t sc = up(G.n * elt), sbx = up((size_t)G.ny * G.nz * elt), sby = up((size_t)G.nx * G.nz * elt);
        const size_t sbz = up((size_t)G.nx * G.ny * elt);
        mem.alloc(3 * sc + sbx + sby + sbz);
        char* p = mem.as<char>();
        L.cx = (const TC*)p;
        L.cy = (const TC*)(p + sc);
        L.cz = (const TC*)(p + 2 * sc);
        L.bxm = (const TC*)(p + 3 * sc);
        L.bym = (const TC*)(p + 3 * sc + sbx);
        L.bzm = (const TC*)(p + 3 * sc + sbx + sby);
    }
};

template <class TC>
static void launch_faces(cudaStream_t s, const Geom& G, const double* K, const mf3d_bc& bc, double scale,
                         const LevelOp<TC>& L) {
    const ColLaunch cl = col_launch(G.nx, G.ny, G.nz);
    faces_kernel<TC><<<cl.grid, cl.block, 0, s>>>(G.nx, G.ny, G.nz, K, to_dev(bc), scale, (TC*)L.cx, (TC*)L.cy,
                                                  (TC*)L.cz, (TC*)L.bxm, (TC*)L.bym, (TC*)L.bzm, cl.zchunk);
    MF3D_LAUNCH_CK();
}

// Power-of-two scale for a bf16 level: 2^-round(log2 of the level's typical coefficient)
// keeps the stored values centred on 1 (bf16 has float's exponent range, so the scale is a
// tested variant, not a range fix).
static double bf16_scale(const Geom& G) {
    (void)G;
    return 1.0;
}

// ---------------------------------------------------------------------------------------
// V-cycle program for levels [0, Lt) in precision (T, TC) plus the FP64 tail [Lt, nl)
// ---------------------------------------------------------------------------------------
struct Timer {
    cudaEvent_t e0, e1;
    cudaStream_t s;
    template <class F> float mean_ms(int reps, F&& f) {
        f(); // warm-up launch
        MF3D_CK(cudaEventRecord(e0, s));
        for (int i = 0; i < reps; ++i) f();
        MF3D_CK(cudaEventRecord(e1, s));
        MF3D_CK(cudaEventSynchronize(e1));
        float ms = 0.f;
        MF3D_CK(cudaEventElapsedTime(&ms, e0, e1));
        return ms / reps;
    }
};

static mf3d_kernel_timing timing(const char* name, float ms, double bytes, int per_iter) {
    mf3d_kernel_timing t{};
    std::snprintf(t.name, sizeof(t.name), "%s", name);
    t.ms = ms;
    t.bytes = bytes;
    t.launches_per_iter = per_iter;
    return t;
}

struct VCycleBase {
    virtual ~VCycleBase() {}
    virtual void build_coefs(cudaStream_t s, const std::vector<const double*>& Klev) = 0;
    // z (type T) = V-cycle of the level-0 right-hand side bound at construction; when
    // rho_out != null, <r64, z> is summed into *rho_out.
    virtual void run(cudaStream_t s, void* z, double* rho_out) = 0;
    // per-kernel timings of one V-cycle (level-0 sweeps by role, the coarse tail, the whole cycle)
    virtual void profile(Timer& tm, int reps, void* z, double* rho_out, std::vector<mf3d_kernel_timing>& out) = 0;
    virtual size_t z_elt() const = 0;
    virtual size_t bytes() const = 0;
    virtual int tma_levels() const = 0;
};

struct Scratch {
    double* partials;
    unsigned* tickets; // one per reduction site
    size_t partial_cap;
    int* err;          // device error flag of the TMA pipelines
};

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link against libcuda).
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        MF3D_CK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || !p) throw Error(MF3D_E_CUDA, "cuTensorMapEncodeTiled unavailable");
        fn = (EncodeTiledFn)p;
    }
    return fn;
}

template <class E> static CUtensorMapDataType tma_dtype();
template <> CUtensorMapDataType tma_dtype<double>() { return CU_TENSOR_MAP_DATA_TYPE_FLOAT64; }
template <> CUtensorMapDataType tma_dtype<float>() { return CU_TENSOR_MAP_DATA_TYPE_FLOAT32; }
template <> CUtensorMapDataType tma_dtype<__nv_bfloat16>() { return CU_TENSOR_MAP_DATA_TYPE_BFLOAT16; }

// 3-D tiled map over an nx*ny*nz array, box bx*by*1; out-of-range elements read as zero.
template <class E> static CUtensorMap make_map(const void* base, const Geom& g, int bx, int by) {
    if (((uintptr_t)base & 15) || ((size_t)g.nx * sizeof(E)) % 16)
        throw Error(MF3D_E_INVALID, "array not aligned for TMA");
    CUtensorMap m;
    cuuint64_t dims[3] = {(cuuint64_t)g.nx, (cuuint64_t)g.ny, (cuuint64_t)g.nz};
    cuuint64_t strides[2] = {(cuuint64_t)g.nx * sizeof(E), (cuuint64_t)g.nx * g.ny * sizeof(E)};
    cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1u};
    cuuint32_t es[3] = {1u, 1u, 1u};
    CUresult r = encode_fn()(&m, tma_dtype<E>(), 3, const_cast<void*>(base), dims, strides, box, es,
                             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw Error(MF3D_E_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
    return m;
}

// 2-D tiled map over a d0*d1 array (the boundary-face planes), box b0*b1.
template <class E> static CUtensorMap make_map2(const void* base, int d0, int d1, int b0, int b1) {
    if (((uintptr_t)base & 15) || ((size_t)d0 * sizeof(E)) % 16)
        throw Error(MF3D_E_INVALID, "array not aligned for TMA");
    CUtensorMap m;
    cuuint64_t dims[2] = {(cuuint64_t)d0, (cuuint64_t)d1};
    cuuint64_t strides[1] = {(cuuint64_t)d0 * sizeof(E)};
    cuuint32_t box[2] = {(cuuint32_t)b0, (cuuint32_t)b1};
    cuuint32_t es[2] = {1u, 1u};
    CUresult r = encode_fn()(&m, tma_dtype<E>(), 2, const_cast<void*>(base), dims, strides, box, es,
                             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                             CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw Error(MF3D_E_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
    return m;
}

// Whether the x-pair sweep stages a level by TMA: no periodic axis, and rows of the arrays
// and of the boundary-face planes that are whole multiples of 16 bytes (a box row of
// cp.async.bulk.tensor starts on a 16-byte boundary).
template <class T, class TC = T> static bool sp_tma_ok(const Geom& g, const mf3d_bc& bc) {
    if (bc.type[0] == MF3D_BC_PERIODIC || bc.type[2] == MF3D_BC_PERIODIC || bc.type[4] == MF3D_BC_PERIODIC)
        return false;
    return g.nx % 2 == 0 && ((size_t)g.nx * sizeof(T)) % 16 == 0 && ((size_t)g.ny * sizeof(T)) % 16 == 0 &&
           ((size_t)g.nx * sizeof(TC)) % 16 == 0 && ((size_t)g.ny * sizeof(TC)) % 16 == 0;
}
// Tensor maps of the TMA-staged x-pair sweep of one level (x: the sweep's input buffer).
template <class T, class TC>
static SpMaps make_sp_maps(const Geom& g, const T* x, const T* b, const LevelOp<TC>& op) {
    using G = SpGeom<T, TC, true>;
    SpMaps m;
    m.x = make_map<T>(x, g, G::W, SP_XR);
    m.b = make_map<T>(b, g, G::W, SP_CR);
    m.cx = make_map<TC>(op.cx, g, G::W, SP_CR);
    m.cy = make_map<TC>(op.cy, g, G::W, SP_YR);
    m.cz = make_map<TC>(op.cz, g, G::W, SP_CR);
    m.bxm = make_map2<TC>(op.bxm, g.ny, g.nz, G::BXN, 1);
    m.bym = make_map2<TC>(op.bym, g.nx, g.nz, G::W, 1);
    m.bzm = make_map2<TC>(op.bzm, g.nx, g.ny, G::W, SP_CR);
    return m;
}

// ---- the coarse levels in one thread-block cluster (kernels_coarse.cuh) ----
struct CoarsePlan {
    int Lc = -1; // first level of the cluster kernel; -1: the one-CTA tail serves the coarse end
    int cn = 0;  // CTAs of the cluster
    size_t smem = 0;
    CoarseArgs a{}; // weights unset
};

// Shared-memory layout of levels Lc .. coarsest with cn CTAs; false when a level does not qualify
// or the layout does not fit.
static bool coarse_layout(const std::vector<Geom>& G, const std::vector<LevelOp<double>>& op, int Lc, int cn,
                          CoarsePlan& p) {
    const int nl = (int)G.size(), nlev = nl - Lc;
    if (nlev < 1 || nlev > TAIL2_MAX_LEVELS) return false;
    CoarseArgs a{};
    a.nlev = nlev;
    int ncl = 0;
    for (int l = Lc; l < nl; ++l) {
        if (G[l].n > (size_t)CT_MAX_CELLS) return false;
        if ((op[l].per_x && G[l].nx % 2) || (op[l].per_y && G[l].ny % 2) || (op[l].per_z && G[l].nz % 2)) return false;
        if (G[l].n > (size_t)CT_LOCAL_MAX) {
            if (ncl != l - Lc) return false; // clustered levels come first
            ++ncl;
        }
    }
    a.ncl = ncl;
    const int last = Lc + ncl - 1; // last clustered level
    int units = 1;
    if (ncl > 0) {
        units = last + 1 < nl ? G[last + 1].nz : G[last].nz;
        if (units < cn) return false;
    } else if (cn != 1) {
        return false;
    }
    a.units = units;
    size_t off = 0;
    for (int l = Lc; l < nl; ++l) {
        CLevel& L = a.L[l - Lc];
        L.nx = G[l].nx;
        L.ny = G[l].ny;
        L.nz = G[l].nz;
        L.n = (int)G[l].n;
        L.per_x = op[l].per_x;
        L.per_y = op[l].per_y;
        L.per_z = op[l].per_z;
        L.clustered = l <= last;
        if (L.clustered) {
            L.shift = last + 1 < nl ? last + 1 - l : last - l;
            if (((long long)units << L.shift) != L.nz) return false;
            L.pmax = ((units + cn - 1) / cn) << L.shift;
        } else {
            L.shift = 0;
            L.pmax = L.nz;
        }
        L.hcap = (L.nx + 1) / 2 * L.ny * L.pmax;
        L.xoff = (int)off;
        off += (size_t)(L.nx + 2) * (L.ny + 2) * (L.pmax + 2);
        L.boff = (int)off;
        off += (size_t)2 * L.hcap;
        L.woff = (int)off;
        off += (size_t)16 * L.hcap;
        L.fhx = make_fdiv((L.nx + 1) / 2);
        L.fnx = make_fdiv(L.nx);
        L.fny = make_fdiv(L.ny);
    }
    {
        const CLevel& C = a.L[nlev - 1];
        if (!C.clustered && C.n <= CT_MAP_MAX) { // coarsest level solved by its map
            a.moff = (int)off;
            off += (size_t)C.n * 2 * C.hcap;
        } else {
            a.moff = -1;
        }
    }
    if (off * sizeof(double) > kCoarseSmemMax) return false;
    p.a = a;
    p.smem = off * sizeof(double);
    p.cn = cn;
    p.Lc = Lc;
    return true;
}

static void coarse_kernel_attrs() {
    static std::once_flag once;
    std::call_once(once, [] {
        MF3D_CK(cudaFuncSetAttribute(coarse_cluster_kernel<float, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)kCoarseSmemMax));
        MF3D_CK(cudaFuncSetAttribute(coarse_cluster_kernel<double, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)kCoarseSmemMax));
        MF3D_CK(cudaFuncSetAttribute(coarse_cluster_kernel<double, double>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCoarseSmemMax));
    });
}

// whether a cluster of cn CTAs with this much shared memory can run on the device
static bool coarse_cluster_fits(int cn, size_t smem) {
    coarse_kernel_attrs();
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)cn);
    cfg.blockDim = dim3(CT_NT);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)cn;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int nc = 0;
    const cudaError_t e = cudaOccupancyMaxActiveClusters(&nc, coarse_cluster_kernel<double, double>, &cfg);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return nc >= 1;
}

// The lowest first level (most levels) for which the cluster kernel works, with the largest
// cluster (a power of two, at most CT_MAX_CLUSTER) that fits; Lc = -1 when none does.
// MF3D_NO_CLUSTER_TAIL=1 keeps the one-CTA tail.
static CoarsePlan plan_coarse(const std::vector<Geom>& G, const std::vector<LevelOp<double>>& op, int Lt) {
    CoarsePlan best;
    if (std::getenv("MF3D_NO_CLUSTER_TAIL")) return best;
    const int nl = (int)G.size();
    int lo = nl - 1;
    while (lo > 0 && G[lo - 1].n <= (size_t)CT_MAX_CELLS) --lo;
    for (int Lc = lo; Lc <= Lt && Lc < nl; ++Lc)
        for (int cn = CT_MAX_CLUSTER; cn >= 1; cn /= 2) {
            CoarsePlan p;
            if (coarse_layout(G, op, Lc, cn, p) && coarse_cluster_fits(cn, p.smem)) return p;
        }
    return best;
}

template <class TI, class TO>
static void launch_coarse(cudaStream_t s, const CoarsePlan& p, const CoarseArgs& a, const TI* b_in, TO* x_out) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)p.cn);
    cfg.blockDim = dim3(CT_NT);
    cfg.dynamicSmemBytes = p.smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)p.cn;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    MF3D_CK(cudaLaunchKernelEx(&cfg, coarse_cluster_kernel<TI, TO>, a, b_in, x_out));
    MF3D_LAUNCH_CK();
}

template <class T, class TC> class VCycle : public VCycleBase {
  public:
    // the x-pair sweep serves FP64 / FP64, FP32 / FP32 and FP32 / BF16 (vector / coefficient)
    static constexpr bool kPair = sizeof(T) == sizeof(TC) ||
                                  (std::is_same<T, float>::value && std::is_same<TC, __nv_bfloat16>::value);

    // b0: level-0 right-hand side in the V-cycle's type (the PCG residual or its FP32 copy);
    // r64: the FP64 residual (dot products, and the right-hand side when the whole V-cycle is
    // the coarse tail).
    // cp: the cluster kernel's plan for single solves (cp.Lc <= Lt), or cp.Lc = -1
    VCycle(const std::vector<Geom>& G, int Lt, const CoarsePlan& cp, const mf3d_bc& bc, bool pin, int pre, int post,
           int coarse, const std::vector<LevelOp<double>>& op64, Scratch scr, const T* b0, const double* r64,
           bool allow_tma)
        : G_(G), Lt_(Lt), cp_(cp), bc_(bc), pin_(pin), pre_(pre), post_(post), coarse_(coarse), op64_(op64),
          scr_(scr), b0_(b0), r64_(r64) {
        const int nl = (int)G.size();
        ops_.resize(Lt);
        coef_.resize(Lt);
        xa_.resize(Lt);
        xb_.resize(Lt);
        bl_.resize(Lt + 1);
        for (int l = 0; l < Lt; ++l) {
            scale_.push_back(std::is_same<TC, __nv_bfloat16>::value ? bf16_scale(G[l]) : 1.0);
            ops_[l] = make_op<TC>(G[l], bc, pin, scale_[l]);
            if (std::is_same<TC, double>::value) {
                // FP64 V-cycle shares the FP64 coefficients
                const LevelOp<double>& o = op64[l];
                ops_[l].cx = (const TC*)o.cx;
                ops_[l].cy = (const TC*)o.cy;
                ops_[l].cz = (const TC*)o.cz;
                ops_[l].bxm = (const TC*)o.bxm;
                ops_[l].bym = (const TC*)o.bym;
                ops_[l].bzm = (const TC*)o.bzm;
            } else {
                coef_[l].reset(new CoefStore());
                coef_[l]->build<TC>(G[l], sizeof(TC), ops_[l]);
                bytes_ += coef_[l]->mem.bytes;
            }
            xa_[l].reset(new DevMem(G[l].n * sizeof(T)));
            xb_[l].reset(new DevMem(G[l].n * sizeof(T)));
            bytes_ += 2 * G[l].n * sizeof(T);
        }
        for (int l = 1; l <= Lt && l < nl; ++l) {
            bl_[l].reset(new DevMem(G[l].n * sizeof(T)));
            bytes_ += G[l].n * sizeof(T);
        }
        // TMA tensor maps for every level the staged sweep can serve
        tma_.assign(Lt, 0);
        maps_.resize(Lt);
        const bool periodic = bc.type[0] == MF3D_BC_PERIODIC || bc.type[2] == MF3D_BC_PERIODIC ||
                              bc.type[4] == MF3D_BC_PERIODIC;
        for (int l = 0; l < Lt && allow_tma && !periodic; ++l) {
            const Geom& g = G[l];
            // TMA boxes start on 16-byte boundaries, and the staged sweep's 4-cell quads need
            // nx to be a multiple of 4 (a quad is all inside the grid or all outside)
            if ((g.nx * sizeof(T)) % 16 || (g.nx * sizeof(TC)) % 16 || (g.ny * sizeof(TC)) % 16 || g.nx % 4 ||
                g.nx < 16 || g.ny < 8)
                continue;
            tma_[l] = 1;
            ++n_tma_;
            for (int resid = 0; resid < 2; ++resid) {
                // box shapes of the staged sweep: x (BX x BY), b / cx / cz (BX x BYC), cy (BX x BYY)
                const int bx = resid ? TmaSweepCfg<T, TC, M_RESID>::BX : TmaSweepCfg<T, TC, 0>::BX;
                const int by = resid ? TmaSweepCfg<T, TC, M_RESID>::BY : TmaSweepCfg<T, TC, 0>::BY;
                const int byc = resid ? TmaSweepCfg<T, TC, M_RESID>::BYC : TmaSweepCfg<T, TC, 0>::BYC;
                const int byy = resid ? TmaSweepCfg<T, TC, M_RESID>::BYY : TmaSweepCfg<T, TC, 0>::BYY;
                Maps4& m = maps_[l][resid];
                const T* b = l == 0 ? b0_ : (const T*)bl_[l]->p;
                m.xa.x = make_map<T>(xa_[l]->p, g, bx, by);
                m.xa.b = make_map<T>(b, g, bx, byc);
                m.xa.cx = make_map<TC>(ops_[l].cx, g, bx, byc);
                m.xa.cy = make_map<TC>(ops_[l].cy, g, bx, byy);
                m.xa.cz = make_map<TC>(ops_[l].cz, g, bx, byc);
                m.xa.bxm = make_map2<TC>(ops_[l].bxm, g.ny, g.nz, TmaSweepCfg<T, TC, 0>::BYP, 1);
                m.xa.bym = make_map2<TC>(ops_[l].bym, g.nx, g.nz, bx, 1);
                m.xa.bzm = make_map2<TC>(ops_[l].bzm, g.nx, g.ny, bx, byc);
                m.xb = m.xa;
                m.xb.x = make_map<T>(xb_[l]->p, g, bx, by);
            }
        }
        if (n_tma_) set_tma_smem();
        // levels the x-pair sweep serves (single solves, every mode but the fused residual):
        // the FP64 V-cycle wherever nx is even and a periodic axis is a whole number of tiles
        // (TMA staging where the grid allows it, cp.async otherwise); the FP32 V-cycle, with FP32
        // or BF16 coefficients, where TMA staging applies (else the quad sweep)
        pair_.assign(Lt, 0);
        pair_tm_.assign(Lt, 0);
        pmaps_.resize(Lt);
        if constexpr (kPair) {
            for (int l = 0; l < Lt; ++l) {
                const Geom& g = G[l];
                if (g.nx % 2) continue;
                if (bc.type[0] == MF3D_BC_PERIODIC && g.nx % SP_TX) continue;
                if (bc.type[2] == MF3D_BC_PERIODIC && g.ny % SP_TY) continue;
                const bool tm = allow_tma && sp_tma_ok<T, TC>(g, bc);
                if (sizeof(T) == 4 && !tm) continue;
                pair_[l] = 1;
                ++n_pair_;
                if (tm) { // TMA staging; maps for both x buffers
                    const T* b = l == 0 ? b0_ : (const T*)bl_[l]->p;
                    pmaps_[l][0] = make_sp_maps<T, TC>(g, (const T*)xa_[l]->p, b, ops_[l]);
                    pmaps_[l][1] = make_sp_maps<T, TC>(g, (const T*)xb_[l]->p, b, ops_[l]);
                    pair_tm_[l] = 1;
                }
            }
            if (n_pair_) set_pair_smem();
        }
        // coarse tail: FP64 weights per cell, x (ghost-padded) and b in shared memory
        if (Lt < nl) {
            tail_.nlev = nl - Lt;
            if (tail_.nlev > TAIL2_MAX_LEVELS) throw Error(MF3D_E_INVALID, "too many coarse tail levels");
            tail_.pre = pre;
            tail_.post = post;
            tail_.coarse_iters = coarse;
            // weights of every level either coarse kernel serves: [Lw, coarsest)
            Lw_ = cp_.Lc >= 0 ? std::min(cp_.Lc, Lt) : Lt;
            size_t wtot = 0;
            for (int l = Lw_; l < nl; ++l) wtot += 8 * G[l].n;
            tail_w_.reset(new DevMem(wtot * sizeof(double)));
            bytes_ += tail_w_->bytes;
            {
                size_t wo = 0;
                for (int l = Lw_; l < nl; ++l) {
                    if (cp_.Lc >= 0 && l >= cp_.Lc) cp_.a.L[l - cp_.Lc].w = tail_w_->as<double>() + wo;
                    wo += 8 * G[l].n;
                }
                if (cp_.Lc >= 0) {
                    cp_.a.pre = pre;
                    cp_.a.post = post;
                    cp_.a.coarse_iters = coarse;
                    cp_.a.M = nullptr;
                    if (cp_.a.moff >= 0) {
                        const CLevel& C = cp_.a.L[cp_.a.nlev - 1];
                        cmap_.reset(new DevMem((size_t)C.n * 2 * C.hcap * sizeof(double)));
                        bytes_ += cmap_->bytes;
                        cp_.a.M = cmap_->as<double>();
                    }
                    if (cp_.Lc > 0 && cp_.Lc < Lt) {
                        ctail_out_.reset(new DevMem(G[cp_.Lc].n * sizeof(T)));
                        bytes_ += ctail_out_->bytes;
                    }
                }
            }
            int off = 0;
            size_t woff = 0;
            for (int l = Lw_; l < Lt; ++l) woff += 8 * G[l].n;
            for (int l = Lt; l < nl; ++l) {
                TailLevel& T2 = tail_.L[l - Lt];
                T2.nx = G[l].nx;
                T2.ny = G[l].ny;
                T2.nz = G[l].nz;
                T2.n = (int)G[l].n;
                T2.per_x = op64[l].per_x;
                T2.per_y = op64[l].per_y;
                T2.per_z = op64[l].per_z;
                T2.xoff = off;
                off += (G[l].nx + 2) * (G[l].ny + 2) * (G[l].nz + 2);
                T2.boff = off;
                off += (int)G[l].n;
                T2.w = tail_w_->as<double>() + woff;
                woff += 8 * G[l].n;
            }
            tail_smem_ = (size_t)off * sizeof(double);
            tail_out_.reset(new DevMem(G[Lt].n * sizeof(T)));
            bytes_ += G[Lt].n * sizeof(T);
            // the attribute belongs to the kernel, not to this solver: set it to the largest
            // tail any solver may have, so that a solver created later with a smaller tail does
            // not lower it under this one
            if (tail_smem_ > kTailSmemMax) throw Error(MF3D_E_INVALID, "coarse tail exceeds shared memory");
            MF3D_CK(cudaFuncSetAttribute(tail2_kernel<T, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kTailSmemMax));
            MF3D_CK(cudaFuncSetAttribute(tail2_kernel<double, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kTailSmemMax));
        }
    }

    // ---- batched solves: run() with rec_ / rec_tail_ set records its sweeps and its coarse
    // tail instead of launching them ----
    struct RecSweep {
        int phase, level, sw, mode; // phase 0: down (pre-smoothing), 1: up (post-smoothing)
        bool tma;                   // the staged (TMA) form exists
        TmaSweepArgs<T, TC> ta;     // staged form, z chunk unset
        const TmaMaps* maps;
        SweepArgs<T, TC, T> la; // L1 form, z chunk unset
        Geom g;
        bool pair;            // the x-pair sweep's TMA form serves this sweep
        SpArgs<T, TC> pa;     // its arguments, z chunk unset
        const SpMaps* pmaps;  // its tensor maps
        int kind;             // 0: a sweep; 1: the residual + restriction after the last pre-sweep
        RrItem<T, TC> rr;     // kind 1: its arguments and grid
    };
    struct RecTail {
        Tail2Args a;
        const T* b;
        T* out;
        size_t smem;
    };
    std::vector<RecSweep>* rec_ = nullptr;
    RecTail* rec_tail_ = nullptr;
    int rec_phase_ = 0, rec_sw_ = 0;
    int levels_above_tail() const { return Lt_; }
    const Scratch& scratch() const { return scr_; }
    int pre() const { return pre_; }
    int post() const { return post_; }

    void build_coefs(cudaStream_t s, const std::vector<const double*>& Klev) override {
        if (!std::is_same<TC, double>::value)
            for (int l = 0; l < Lt_; ++l) launch_faces<TC>(s, G_[l], Klev[l], bc_, scale_[l], ops_[l]);
        size_t wo = 0;
        for (int l = Lw_; l < (int)G_.size(); ++l) {
            tail_weights_kernel<<<grid1d(G_[l].n, 256), 256, 0, s>>>(op64_[l], tail_w_->as<double>() + wo);
            MF3D_LAUNCH_CK();
            wo += 8 * G_[l].n;
        }
        if (cmap_) { // the coarsest level's sweeps as a matrix, one column per cell
            const int nl = (int)G_.size();
            const CLevel& C = cp_.a.L[cp_.a.nlev - 1];
            MF3D_CK(cudaMemsetAsync(cmap_->p, 0, cmap_->bytes, s));
            coarse_map_kernel<<<C.n, 64, 0, s>>>(tail_.L[nl - 1 - Lt_], C, coarse_, cmap_->as<double>());
            MF3D_LAUNCH_CK();
        }
    }

    size_t z_elt() const override { return sizeof(T); }
    size_t bytes() const override { return bytes_; }
    int tma_levels() const override { return n_tma_; }

    void run(cudaStream_t s, void* zv, double* rho_out) override {
        T* z = (T*)zv;
        const int nl = (int)G_.size();
        // levels above the coarse kernel: the cluster kernel's for single solves, the one-CTA
        // tail's for batched ones
        const int Lb = coarse_start();
        std::vector<const T*> cur(Lb + 1, nullptr), fin(Lb + 1, nullptr);
        // ---- down ----
        for (int l = 0; l < Lb; ++l) {
            T* bc_next = (T*)bl_[l + 1]->p;
            const T* c = nullptr;
            for (int sw = 1; sw <= pre_; ++sw) {
                T* out = other(l, c);
                int mode = (c ? 0 : M_ZERO) | (sw == pre_ ? M_RESID : 0);
                rec_phase_ = 0;
                rec_sw_ = 2 * sw; // (2 sw + 1: the residual + restriction after it)
                // staged levels: the last pre-sweep, then the residual and its restriction in a
                // kernel of their own (batched solves record the fused form)
                const bool split = (mode & M_RESID) && (tma_[l] || pair_[l]) && split_resid_ && !rec_;
                sweep(s, l, c, out, nullptr, split ? nullptr : bc_next, split ? (mode & ~M_RESID) : mode, nullptr);
                if (split) resid_restrict(s, l, out, bc_next);
                c = out;
            }
            if (pre_ == 0) restrict_b(s, l, bc_next);
            cur[l] = c;
        }
        // ---- coarse end (FP64): one cluster, or one CTA ----
        const T* e_below = nullptr;
        if (Lb < nl) {
            T* out = coarse_out(z);
            launch_tail(s, out);
            e_below = out;
            if (Lb == 0 && rho_out) dot_rz(s, z, G_[0].n, rho_out);
        }
        // ---- up ----
        for (int l = Lb - 1; l >= 0; --l) {
            const T* c = cur[l];
            const T* e = (l + 1 == Lb) ? e_below : fin[l + 1];
            for (int sw = 1; sw <= post_; ++sw) {
                const bool last = sw == post_;
                T* out = (l == 0 && last) ? z : other(l, c);
                int mode = (c ? 0 : M_ZERO) | (sw == 1 ? M_PROLONG : 0) | ((l == 0 && last && rho_out) ? M_DOT : 0);
                rec_phase_ = 1;
                rec_sw_ = 2 * sw; // (2 sw + 1: the residual + restriction after it)
                sweep(s, l, c, out, e, nullptr, mode, rho_out);
                c = out;
            }
            if (post_ == 0) {
                T* out = (l == 0) ? z : other(l, c);
                prolong_kernel<T><<<grid1d(G_[l].n, 256), 256, 0, s>>>(G_[l].nx, G_[l].ny, G_[l].nz, c, e, out);
                MF3D_LAUNCH_CK();
                c = out;
                if (l == 0 && rho_out) dot_rz(s, z, G_[0].n, rho_out);
            }
            fin[l] = c;
        }
    }

    void profile(Timer& tm, int reps, void* zv, double* rho_out, std::vector<mf3d_kernel_timing>& out) override {
        T* z = (T*)zv;
        const int nl = (int)G_.size();
        out.push_back(timing("vcycle_total", tm.mean_ms(reps, [&] { run(tm.s, zv, rho_out); }), 0.0, 1));
        const int Lb = coarse_start();
        if (Lb >= 1) {
            const double n = (double)G_[0].n, et = sizeof(T), ec = sizeof(TC);
            const double coef = 3.0 * n * ec, nc = n / 8.0;
            T* xa = (T*)xa_[0]->p;
            T* xb = (T*)xb_[0]->p;
            T* bc1 = (T*)bl_[1]->p;
            const T* e1 = (coarse_start() == 1) ? (const T*)coarse_out(z) : (const T*)xa_[1]->p;
            const int pre_extra = std::max(0, pre_ - 2), post_extra = std::max(0, post_ - 2);
            const char* tag = pair_[0] ? "pair" : (tma_[0] ? "tma" : "ldg");
            char nm[40];
            if (pre_ >= 1) {
                std::snprintf(nm, sizeof(nm), "sweep_l0_zero_in_%s", tag);
                out.push_back(timing(nm, tm.mean_ms(reps, [&] {
                    sweep(tm.s, 0, nullptr, xa, nullptr, bc1, pre_ == 1 ? (M_ZERO | M_RESID) : M_ZERO, nullptr);
                }), et * n + coef + et * n + (pre_ == 1 ? et * nc : 0.0), 1));
            }
            if (pre_ >= 2 && (tma_[0] || pair_[0]) && split_resid_) {
                std::snprintf(nm, sizeof(nm), "sweep_l0_2nd_pre_%s", tag);
                out.push_back(timing(nm, tm.mean_ms(reps, [&] {
                    sweep(tm.s, 0, xa, xb, nullptr, nullptr, 0, nullptr);
                }), et * n + et * n + coef + et * n, 1));
                out.push_back(timing("resid_restrict_l0", tm.mean_ms(reps, [&] { resid_restrict(tm.s, 0, xb, bc1); }),
                                     et * n + et * n + coef + et * nc, 1));
            } else if (pre_ >= 2) {
                std::snprintf(nm, sizeof(nm), "sweep_l0_resid_restrict_%s", tag);
                out.push_back(timing(nm, tm.mean_ms(reps, [&] {
                    sweep(tm.s, 0, xa, xb, nullptr, bc1, M_RESID, nullptr);
                }), et * n + et * n + coef + et * n + et * nc, 1));
            }
            if (pre_extra + post_extra > 0) {
                std::snprintf(nm, sizeof(nm), "sweep_l0_plain_%s", tag);
                out.push_back(timing(nm, tm.mean_ms(reps, [&] {
                    sweep(tm.s, 0, xa, xb, nullptr, nullptr, 0, nullptr);
                }), et * n + et * n + coef + et * n, pre_extra + post_extra));
            }
            if (post_ >= 2) {
                std::snprintf(nm, sizeof(nm), "sweep_l0_prolong_%s", tag);
                out.push_back(timing(nm, tm.mean_ms(reps, [&] {
                    sweep(tm.s, 0, xb, xa, e1, nullptr, M_PROLONG, nullptr);
                }), et * n + et * nc + et * n + coef + et * n, 1));
            }
            if (post_ >= 1) {
                std::snprintf(nm, sizeof(nm), "sweep_l0_dot_out_%s", tag);
                out.push_back(timing(nm, tm.mean_ms(reps, [&] {
                    sweep(tm.s, 0, xa, z, e1, nullptr, post_ == 1 ? (M_PROLONG | M_DOT) : M_DOT, rho_out);
                }), et * n + et * n + coef + et * n + 8.0 * n + (post_ == 1 ? et * nc : 0.0), 1));
            }
            for (int l = 1; l < Lb; ++l) {
                std::snprintf(nm, sizeof(nm), "sweep_l%d_plain_%s", l, pair_[l] ? "pair" : (tma_[l] ? "tma" : "ldg"));
                T* a = (T*)xa_[l]->p;
                T* b = (T*)xb_[l]->p;
                const double nn = (double)G_[l].n;
                out.push_back(timing(nm, tm.mean_ms(reps, [&] { sweep(tm.s, l, a, b, nullptr, nullptr, 0, nullptr); }),
                                     3.0 * et * nn + 3.0 * nn * ec, pre_ + post_));
            }
        }
        if (Lb < nl) {
            T* outp = coarse_out(z);
            out.push_back(timing(cluster_on() ? "coarse_cluster" : "coarse_tail",
                                 tm.mean_ms(reps, [&] { launch_tail(tm.s, outp); }), 0.0, 1));
        }
    }

  private:
    struct Maps4 {
        TmaMaps xa, xb; // x read from xa or from xb
    };

    T* other(int l, const T* c) const { return (c == (const T*)xa_[l]->p) ? (T*)xb_[l]->p : (T*)xa_[l]->p; }

    // the cluster kernel serves this solve's coarse end (single solves with a plan)
    bool cluster_on() const { return cp_.Lc >= 0 && !rec_tail_ && !rec_; }
    int coarse_start() const { return cluster_on() ? cp_.Lc : Lt_; }
    // where the coarse end writes its correction: z when it is the whole V-cycle
    T* coarse_out(T* z) const {
        const int Lb = coarse_start();
        if (Lb == 0) return z;
        if (cluster_on() && Lb < Lt_) return (T*)ctail_out_->p;
        return (T*)tail_out_->p;
    }

    void launch_tail(cudaStream_t s, T* out) {
        if (cluster_on()) {
            if (cp_.Lc == 0)
                launch_coarse<double, T>(s, cp_, cp_.a, r64_, out);
            else
                launch_coarse<T, T>(s, cp_, cp_.a, (const T*)bl_[cp_.Lc]->p, out);
            return;
        }
        if (rec_tail_) { // batched solve: record only (the batch needs a level above the tail)
            if (Lt_ == 0) throw Error(MF3D_E_INVALID, "batched solve: the whole hierarchy fits the coarse tail");
            rec_tail_->a = tail_;
            rec_tail_->b = (const T*)bl_[Lt_]->p;
            rec_tail_->out = out;
            rec_tail_->smem = tail_smem_;
            return;
        }
        if (Lt_ == 0)
            tail2_kernel<double, T><<<1, TAIL2_NT, tail_smem_, s>>>(tail_, r64_, out);
        else
            tail2_kernel<T, T><<<1, TAIL2_NT, tail_smem_, s>>>(tail_, (const T*)bl_[Lt_]->p, out);
        MF3D_LAUNCH_CK();
    }

    static int zchunk_for(const Geom& g, int nblk_xy, int target_blocks) {
        // about target_blocks CTAs in total, each marching an even number of planes
        int nzc = std::max(1, (int)std::min<long long>(g.nz, std::max(1, target_blocks / std::max(1, nblk_xy))));
        int zc = (g.nz + nzc - 1) / nzc;
        zc = std::max(2, (zc + 1) & ~1);
        return std::min(zc, ((g.nz + 1) & ~1));
    }

    // arguments of the staged (TMA) sweep of level l, but for its z chunk; *maps the tensor
    // maps of the input buffer
    TmaSweepArgs<T, TC> tma_args(int l, const T* x_in, T* x_out, const T* e, T* b_coarse, int mode, double* dot_out,
                                 const TmaMaps** maps) const {
        TmaSweepArgs<T, TC> a{};
        a.L = ops_[l];
        a.x_out = x_out;
        a.e_c = e;
        if (l + 1 < (int)G_.size()) {
            a.ncx = G_[l + 1].nx;
            a.ncy = G_[l + 1].ny;
        }
        a.b_coarse = b_coarse;
        a.r64 = r64_;
        a.dot_partials = scr_.partials;
        a.dot_ticket = scr_.tickets + 0;
        a.dot_out = dot_out;
        a.err = scr_.err;
        const Maps4& m4 = maps_[l][(mode & M_RESID) ? 1 : 0];
        *maps = (x_in == (const T*)xb_[l]->p) ? &m4.xb : &m4.xa;
        if (x_in && x_in != (const T*)xa_[l]->p && x_in != (const T*)xb_[l]->p)
            throw Error(MF3D_E_INVALID, "sweep input is not a level buffer");
        return a;
    }

    // arguments of the L1-path sweep of level l, but for its z chunk
    SweepArgs<T, TC, T> ldg_args(int l, const T* x_in, T* x_out, const T* e, T* b_coarse, double* dot_out) const {
        SweepArgs<T, TC, T> a{};
        a.L = ops_[l];
        a.b = l == 0 ? b0_ : (const T*)bl_[l]->p;
        a.x_in = x_in;
        a.x_out = x_out;
        a.e_c = e;
        if (l + 1 < (int)G_.size()) {
            a.ncx = G_[l + 1].nx;
            a.ncy = G_[l + 1].ny;
        }
        a.b_coarse = b_coarse;
        a.dot_partials = scr_.partials;
        a.dot_ticket = scr_.tickets + 0;
        a.dot_out = dot_out;
        a.r64 = r64_;
        return a;
    }

    void sweep(cudaStream_t s, int l, const T* x_in, T* x_out, const T* e, T* b_coarse, int mode, double* dot_out) {
        const Geom& g = G_[l];
        const bool tma = tma_[l] != 0;
        if (rec_) { // batched solve: record both forms, launch nothing
            RecSweep r{};
            r.phase = rec_phase_;
            r.level = l;
            r.sw = rec_sw_;
            r.mode = mode;
            r.g = g;
            r.tma = tma;
            if (tma) r.ta = tma_args(l, x_in, x_out, e, b_coarse, mode, dot_out, &r.maps);
            r.la = ldg_args(l, x_in, x_out, e, b_coarse, dot_out);
            r.pair = false;
            r.pmaps = nullptr;
            r.kind = 0;
            if constexpr (kPair) {
                if (pair_[l] && pair_tm_[l] && !(mode & M_RESID)) {
                    r.pair = true;
                    r.pa = pair_args(l, x_in, x_out, e, dot_out);
                    r.pmaps = &pair_maps(l, x_in, mode);
                }
            }
            rec_->push_back(r);
            return;
        }
        if constexpr (kPair) {
            if (pair_[l] && !(mode & M_RESID)) {
                pair_sweep(s, l, x_in, x_out, e, mode, dot_out);
                return;
            }
        }
        const int tx = tma ? TmaSweepCfg<T, TC, 0>::TX : SW_TX, ty = tma ? tma_ty() : SW_TY;
        const int gx = (g.nx + tx - 1) / tx, gy = (g.ny + ty - 1) / ty;
        if (tma) {
            // (tile, z chunk) CTAs, all resident at once: the most chunks per tile that fit
            const long long ntiles = (long long)gx * gy;
            const long long resident = (long long)std::max(1, occ_[mode & 15]) * num_sms();
            const int nchunk = (int)std::max<long long>(1, std::min<long long>(g.nz / 2, resident / ntiles));
            const int zc = 2 * (((g.nz + 1) / 2 + nchunk - 1) / nchunk);
            const long long nblk = ntiles * ((g.nz + zc - 1) / zc);
            const dim3 grid((unsigned)std::min(nblk, std::max(resident, ntiles)));
            if ((mode & M_DOT) && grid.x > scr_.partial_cap) throw Error(MF3D_E_INVALID, "reduction scratch too small");
            const TmaMaps* maps = nullptr;
            TmaSweepArgs<T, TC> a = tma_args(l, x_in, x_out, e, b_coarse, mode, dot_out, &maps);
            a.zchunk = zc;
            dispatch_tma(s, grid, mode, *maps, a);
            return;
        }
        const int zc = zchunk_for(g, gx * gy, num_sms() * 6);
        const int gz = (g.nz + zc - 1) / zc;
        dim3 grid(gx, gy, gz);
        const unsigned nblk = (unsigned)gx * gy * gz;
        if ((mode & M_DOT) && nblk > scr_.partial_cap) throw Error(MF3D_E_INVALID, "reduction scratch too small");
        SweepArgs<T, TC, T> a = ldg_args(l, x_in, x_out, e, b_coarse, dot_out);
        a.zchunk = zc;
        dispatch(s, grid, mode, a);
    }

    template <int MODE> void set_one() {
        using C = TmaSweepCfg<T, TC, MODE>;
        MF3D_CK(cudaFuncSetAttribute(sweep_tma_kernel<T, TC, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)C::SMEM));
        // all of the unified L1 as shared memory, so that MINB CTAs are co-resident
        MF3D_CK(cudaFuncSetAttribute(sweep_tma_kernel<T, TC, MODE>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                     (int)cudaSharedmemCarveoutMaxShared));
        int n = 0;
        MF3D_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, sweep_tma_kernel<T, TC, MODE>, C::NT, C::SMEM));
        if (n < 1) throw Error(MF3D_E_CUDA, "staged sweep does not fit on an SM");
        occ_[MODE & 15] = n;
    }
    void set_tma_smem() {
        set_one<0>();
        set_one<M_ZERO>();
        set_one<M_PROLONG>();
        set_one<M_ZERO | M_PROLONG>();
        set_one<M_RESID>();
        set_one<M_ZERO | M_RESID>();
        set_one<M_DOT>();
        set_one<M_ZERO | M_DOT>();
        set_one<M_PROLONG | M_DOT>();
        set_one<M_ZERO | M_PROLONG | M_DOT>();
    }

    static int tma_ty() { return TmaSweepCfg<T, TC, 0>::TY; }

    // ---- the x-pair sweep (kernels_sweep_pair.cuh) ----
    template <int MODE> void set_pair_one() {
        if constexpr (kPair) {
            if constexpr (std::is_same<T, TC>::value) pocc_[MODE & 15] = pair_sweep_setup<T, TC, MODE, false>();
            pocc_tm_[MODE & 15] = pair_sweep_setup<T, TC, MODE, true>();
        }
    }
    void set_pair_smem() {
        set_pair_one<0>();
        set_pair_one<M_ZERO>();
        set_pair_one<M_PROLONG>();
        set_pair_one<M_ZERO | M_PROLONG>();
        set_pair_one<M_DOT>();
        set_pair_one<M_ZERO | M_DOT>();
        set_pair_one<M_PROLONG | M_DOT>();
        set_pair_one<M_ZERO | M_PROLONG | M_DOT>();
    }
    // arguments of the x-pair sweep of level l, but for its z chunk
    SpArgs<T, TC> pair_args(int l, const T* x_in, T* x_out, const T* e, double* dot_out) const {
        SpArgs<T, TC> a{};
        a.L = ops_[l];
        a.x_in = x_in;
        a.b = l == 0 ? b0_ : (const T*)bl_[l]->p;
        a.x_out = x_out;
        a.e_c = e;
        if (l + 1 < (int)G_.size()) {
            a.ncx = G_[l + 1].nx;
            a.ncy = G_[l + 1].ny;
        }
        a.r64 = r64_;
        a.dot_partials = scr_.partials;
        a.dot_ticket = scr_.tickets + 0;
        a.dot_out = dot_out;
        a.err = scr_.err;
        return a;
    }
    // tensor maps of the TMA form of level l for the input buffer x_in
    const SpMaps& pair_maps(int l, const T* x_in, int mode) const {
        if (!(mode & M_ZERO) && x_in != (const T*)xa_[l]->p && x_in != (const T*)xb_[l]->p)
            throw Error(MF3D_E_INVALID, "sweep input is not a level buffer");
        return pmaps_[l][x_in == (const T*)xb_[l]->p ? 1 : 0];
    }
    void pair_sweep(cudaStream_t s, int l, const T* x_in, T* x_out, const T* e, int mode, double* dot_out) {
        if constexpr (kPair) {
            const Geom& g = G_[l];
            SpArgs<T, TC> a = pair_args(l, x_in, x_out, e, dot_out);
            const bool tm = pair_tm_[l] != 0;
            const long long resident = (long long)std::max(1, (tm ? pocc_tm_ : pocc_)[mode & 15]) * num_sms();
            const dim3 grid = pair_grid(g, resident, &a.zchunk, tm ? sp_tx<T, TC, true>() : sp_tx<T, TC, false>());
            if ((mode & M_DOT) && grid.x > scr_.partial_cap) throw Error(MF3D_E_INVALID, "reduction scratch too small");
            static const SpMaps no_maps{};
            const SpMaps& m = !tm ? no_maps : pair_maps(l, x_in, mode);
            launch_pair_sweep<T, TC>(s, grid, mode, tm, m, a);
        }
    }

    template <int MODE>
    static void launch_tma(cudaStream_t s, dim3 grid, const TmaMaps& m, const TmaSweepArgs<T, TC>& a) {
        using C = TmaSweepCfg<T, TC, MODE>;
        sweep_tma_kernel<T, TC, MODE><<<grid, C::NT, C::SMEM, s>>>(m, a);
    }

    void dispatch_tma(cudaStream_t s, dim3 grid, int mode, const TmaMaps& m, const TmaSweepArgs<T, TC>& a) {
        switch (mode) {
        case 0: launch_tma<0>(s, grid, m, a); break;
        case M_ZERO: launch_tma<M_ZERO>(s, grid, m, a); break;
        case M_PROLONG: launch_tma<M_PROLONG>(s, grid, m, a); break;
        case M_ZERO | M_PROLONG: launch_tma<M_ZERO | M_PROLONG>(s, grid, m, a); break;
        case M_RESID: launch_tma<M_RESID>(s, grid, m, a); break;
        case M_ZERO | M_RESID: launch_tma<M_ZERO | M_RESID>(s, grid, m, a); break;
        case M_DOT: launch_tma<M_DOT>(s, grid, m, a); break;
        case M_ZERO | M_DOT: launch_tma<M_ZERO | M_DOT>(s, grid, m, a); break;
        case M_PROLONG | M_DOT: launch_tma<M_PROLONG | M_DOT>(s, grid, m, a); break;
        case M_ZERO | M_PROLONG | M_DOT: launch_tma<M_ZERO | M_PROLONG | M_DOT>(s, grid, m, a); break;
        default: throw Error(MF3D_E_INVALID, "unsupported sweep mode");
        }
        MF3D_LAUNCH_CK();
    }

    void dispatch(cudaStream_t s, dim3 grid, int mode, const SweepArgs<T, TC, T>& a) {
        switch (mode) {
        case 0: sweep_kernel<T, TC, T, 0><<<grid, SW_NT, 0, s>>>(a); break;
        case M_ZERO: sweep_kernel<T, TC, T, M_ZERO><<<grid, SW_NT, 0, s>>>(a); break;
        case M_PROLONG: sweep_kernel<T, TC, T, M_PROLONG><<<grid, SW_NT, 0, s>>>(a); break;
        case M_ZERO | M_PROLONG: sweep_kernel<T, TC, T, M_ZERO | M_PROLONG><<<grid, SW_NT, 0, s>>>(a); break;
        case M_RESID: sweep_kernel<T, TC, T, M_RESID><<<grid, SW_NT, 0, s>>>(a); break;
        case M_ZERO | M_RESID: sweep_kernel<T, TC, T, M_ZERO | M_RESID><<<grid, SW_NT, 0, s>>>(a); break;
        case M_DOT: sweep_kernel<T, TC, T, M_DOT><<<grid, SW_NT, 0, s>>>(a); break;
        case M_ZERO | M_DOT: sweep_kernel<T, TC, T, M_ZERO | M_DOT><<<grid, SW_NT, 0, s>>>(a); break;
        case M_PROLONG | M_DOT: sweep_kernel<T, TC, T, M_PROLONG | M_DOT><<<grid, SW_NT, 0, s>>>(a); break;
        case M_ZERO | M_PROLONG | M_DOT:
            sweep_kernel<T, TC, T, M_ZERO | M_PROLONG | M_DOT><<<grid, SW_NT, 0, s>>>(a);
            break;
        default: throw Error(MF3D_E_INVALID, "unsupported sweep mode");
        }
        MF3D_LAUNCH_CK();
    }

    void resid_restrict(cudaStream_t s, int l, const T* x, T* out) {
        const Geom& g = G_[l];
        const T* b = l == 0 ? b0_ : (const T*)bl_[l]->p;
        if constexpr (sizeof(TC) >= 4 || kPair) { // staged: 32 x 16 tiles of x-pairs, even z chunks
            const int gx = (g.nx + RR_TX - 1) / RR_TX, gy = (g.ny + RR_TY - 1) / RR_TY, ncz = g.nz / 2;
            const long long tiles = (long long)gx * gy;
            const int nzc = (int)std::max<long long>(
                1, std::min<long long>(ncz, (long long)num_sms() * MF3D_RR_PERSM / std::max(1LL, tiles)));
            const int zc = 2 * ((ncz + nzc - 1) / nzc);
            const dim3 grid(gx, gy, (g.nz + zc - 1) / zc);
            if (rec_) { // batched solve: record only
                RecSweep r{};
                r.phase = rec_phase_;
                r.level = l;
                r.sw = rec_sw_ + 1;
                r.mode = -1;
                r.g = g;
                r.kind = 1;
                r.rr.L = ops_[l];
                r.rr.x = x;
                r.rr.b = b;
                r.rr.out = out;
                r.rr.zchunk = zc;
                r.rr.gx = (int)grid.x;
                r.rr.gy = (int)grid.y;
                r.rr.gz = (int)grid.z;
                rec_->push_back(r);
                return;
            }
            MF3D_CK(cudaFuncSetAttribute(resid_restrict_staged_kernel<T, TC>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rr_smem_bytes<T, TC>()));
            resid_restrict_staged_kernel<T, TC><<<grid, 256, rr_smem_bytes<T, TC>(), s>>>(ops_[l], x, b, out, zc);
            MF3D_LAUNCH_CK();
        } else {
            throw Error(MF3D_E_INVALID, "the separate residual kernel needs 4- or 8-byte coefficients");
        }
    }

    void restrict_b(cudaStream_t s, int l, T* out) {
        const Geom& c = G_[l + 1];
        const T* fine = l == 0 ? b0_ : (const T*)bl_[l]->p;
        restrict_kernel<T, T><<<grid1d(c.n, 256), 256, 0, s>>>(c.nx, c.ny, c.nz, fine, out);
        MF3D_LAUNCH_CK();
    }

    void dot_rz(cudaStream_t s, const T* z, size_t n, double* out);

    std::vector<Geom> G_;
    int Lt_;
    CoarsePlan cp_; // the cluster kernel (cp_.Lc >= 0) for single solves
    mf3d_bc bc_;
    bool pin_;
    int pre_, post_, coarse_;
    std::vector<LevelOp<double>> op64_;
    Scratch scr_;
    const T* b0_;
    const double* r64_;
    std::vector<LevelOp<TC>> ops_;
    std::vector<double> scale_;
    std::vector<std::unique_ptr<CoefStore>> coef_;
    std::vector<std::unique_ptr<DevMem>> xa_, xb_, bl_;
    std::vector<int> tma_;
    std::vector<std::array<Maps4, 2>> maps_;
    int n_tma_ = 0;
    // Staged levels: the residual and its restriction in a kernel of their own
    // (resid_restrict_staged_kernel) after the last pre-sweep, which computes every cell's
    // residual exactly and is faster than the fused RESID sweep (measured at 256^3 in FP32:
    // 0.152 + 0.069 ms against 0.280 ms).  Batched solves keep the fused sweep.
    static constexpr bool split_resid_ = sizeof(TC) >= 4 || kPair;
    int occ_[16] = {}; // resident staged-sweep CTAs per SM, by mode
    std::vector<int> pair_;    // levels served by the x-pair sweep
    std::vector<int> pair_tm_; // ... with TMA staging
    std::vector<std::array<SpMaps, 2>> pmaps_; // their tensor maps, x read from xa / xb
    int n_pair_ = 0;
    int pocc_[16] = {}, pocc_tm_[16] = {}; // resident x-pair-sweep CTAs per SM, by mode
    std::unique_ptr<DevMem> tail_out_, tail_w_, ctail_out_, cmap_;
    Tail2Args tail_{};
    int Lw_ = 0; // first level with FP64 weights
    size_t tail_smem_ = 0;
    size_t bytes_ = 0;
};

template <class T>
__global__ void dot_kernel(size_t n, const double* __restrict__ a, const T* __restrict__ b, double* partials,
                           unsigned* ticket, double* out) {
    double acc = 0.0;
    for (size_t c = blockIdx.x * (size_t)PK_NT + threadIdx.x; c < n; c += (size_t)gridDim.x * PK_NT)
        acc += a[c] * (double)b[c];
    double v[1] = {acc}, o[1];
    if (grid_sums<PK_NT, 1>(v, partials, ticket, gridDim.x, o)) *out = o[0];
}

template <class T, class TC>
void VCycle<T, TC>::dot_rz(cudaStream_t s, const T* z, size_t n, double* out) {
    const unsigned nb = std::min<unsigned>(grid1d(n, PK_NT), (unsigned)scr_.partial_cap);
    dot_kernel<T><<<nb, PK_NT, 0, s>>>(n, r64_, z, scr_.partials, scr_.tickets + 1, out);
    MF3D_LAUNCH_CK();
}

template <class T, class TC> class BatchSolverT;

// ---------------------------------------------------------------------------------------
// HeadSolver
// ---------------------------------------------------------------------------------------
class HeadSolver {
    template <class T, class TC> friend class BatchSolverT;

  public:
    HeadSolver(const mf3d_grid& g, const mf3d_bc& bc, const mf3d_solver_config& cfg, cudaStream_t user_stream)
        : grid_(g), bc_(bc), cfg_(cfg) {
        if (g.nx < 2 || g.ny < 2 || g.nz < 2) throw Error(MF3D_E_INVALID, "grid must have at least 2 cells per axis");
        if (!(g.dx > 0)) throw Error(MF3D_E_INVALID, "dx must be positive");
        validate_bc(bc);
        if (cfg.solver != MF3D_SOLVER_PCG_MG && cfg.solver != MF3D_SOLVER_MG && cfg.solver != MF3D_SOLVER_CG)
            throw Error(MF3D_E_INVALID, "unknown solver type");
        if (cfg.mg_pre_smooth < 0 || cfg.mg_post_smooth < 0 || cfg.mg_coarse_iters < 0 || cfg.cg_max_iter < 0)
            throw Error(MF3D_E_INVALID, "negative iteration count");
        for (int a = 0; a < 3; ++a) {
            const int n = a == 0 ? g.nx : (a == 1 ? g.ny : g.nz);
            if (bc.type[2 * a] == MF3D_BC_PERIODIC && (n & 1))
                throw Error(MF3D_E_INVALID, "red-black smoothing needs an even cell count on a periodic axis");
        }
        pin_ = pin_enabled(cfg.pin_mode, bc);
        G_ = make_levels(g, cfg.mg_levels);
        const int nl = (int)G_.size();
        // coarse tail: the levels of at most 4096 cells whose padded x and b fit in shared memory
        auto tail_bytes = [&](int l) {
            return (size_t)8 * ((size_t)(G_[l].nx + 2) * (G_[l].ny + 2) * (G_[l].nz + 2) + G_[l].n);
        };
        Lt_ = nl - 1;
        size_t tbytes = tail_bytes(nl - 1);
        while (Lt_ > 0 && G_[Lt_ - 1].n <= 4096 && tbytes + tail_bytes(Lt_ - 1) <= kTailSmemMax) {
            --Lt_;
            tbytes += tail_bytes(Lt_);
        }
        if (tbytes > kTailSmemMax)
            throw Error(MF3D_E_INVALID, "coarsest level too large for the coarse solver (raise mg_levels)");
        if (user_stream) {
            stream_ = user_stream;
        } else {
            MF3D_CK(cudaStreamCreateWithFlags(&own_stream_, cudaStreamNonBlocking));
            stream_ = own_stream_;
        }
        const size_t n = G_[0].n;
        // FP64 operator coefficients: level 0 (PCG operator), tail levels, and every level of an
        // FP64 V-cycle.
        op64_.resize(nl);
        coef64_.resize(nl);
        for (int l = 0; l < nl; ++l) op64_[l] = make_op<double>(G_[l], bc, pin_, 1.0);
        // the coarse levels of single solves in one thread-block cluster, where they qualify
        cplan_ = plan_coarse(G_, op64_, Lt_);
        const int Lw = cplan_.Lc >= 0 ? std::min(cplan_.Lc, Lt_) : Lt_;
        for (int l = 0; l < nl; ++l) {
            if (l == 0 || l >= Lw || cfg.precision == MF3D_PREC_FP64) {
                coef64_[l].reset(new CoefStore());
                coef64_[l]->build<double>(G_[l], sizeof(double), op64_[l]);
                bytes_ += coef64_[l]->mem.bytes;
            }
        }
        Klev_.resize(nl);
        for (int l = 0; l < nl; ++l) {
            Klev_[l].reset(new DevMem(G_[l].n * sizeof(double)));
            bytes_ += G_[l].n * sizeof(double);
        }
        auto vec = [&](DevMem& m) {
            m.alloc(n * sizeof(double));
            MF3D_CK(cudaMemsetAsync(m.p, 0, m.bytes, stream_));
            bytes_ += m.bytes;
        };
        vec(x_);
        vec(b_);
        vec(r_);
        vec(p_);
        vec(p2_);
        vec(Ap_);
        vec(x0_);
        // reduction scratch sized for the largest grid any reduction uses
        size_t cap = std::max<size_t>((size_t)grid1d(n, PK_NT) * 2, col_launch(G_[0].nx, G_[0].ny, G_[0].nz).nblocks) + 1024;
        {
            const int gx = (G_[0].nx + SW_TX - 1) / SW_TX, gy = (G_[0].ny + SW_TY - 1) / SW_TY;
            cap = std::max(cap, (size_t)gx * gy * (size_t)((G_[0].nz + 7) / 8) + 1024);
        }
        partials_.alloc(cap * 2 * sizeof(double));
        tickets_.alloc(16 * sizeof(unsigned));
        state_.alloc(sizeof(PcgState));
        mb_.alloc(4 * sizeof(double));
        MF3D_CK(cudaMemsetAsync(tickets_.p, 0, tickets_.bytes, stream_));
        MF3D_CK(cudaMemsetAsync(state_.p, 0, state_.bytes, stream_));
        bytes_ += partials_.bytes;
        err_.alloc(sizeof(int) * 4);
        MF3D_CK(cudaMemsetAsync(err_.p, 0, err_.bytes, stream_));
        Scratch scr{partials_.as<double>(), tickets_.as<unsigned>() + 8, cap, err_.as<int>()};
        const int prec = cfg.precision;
        const bool tma = std::getenv("MF3D_NO_TMA") == nullptr;
        if (prec != MF3D_PREC_FP64) {
            r32_.alloc(n * sizeof(float));
            bytes_ += r32_.bytes;
        }
        if (prec == MF3D_PREC_FP64)
            vc_.reset(new VCycle<double, double>(G_, Lt_, cplan_, bc, pin_, cfg.mg_pre_smooth, cfg.mg_post_smooth,
                                                 cfg.mg_coarse_iters, op64_, scr, r_.as<double>(), r_.as<double>(), tma));
        else if (prec == MF3D_PREC_FP32)
            vc_.reset(new VCycle<float, float>(G_, Lt_, cplan_, bc, pin_, cfg.mg_pre_smooth, cfg.mg_post_smooth,
                                               cfg.mg_coarse_iters, op64_, scr, r32_.as<float>(), r_.as<double>(), tma));
        else if (prec == MF3D_PREC_BF16)
            vc_.reset(new VCycle<float, __nv_bfloat16>(G_, Lt_, cplan_, bc, pin_, cfg.mg_pre_smooth, cfg.mg_post_smooth,
                                                       cfg.mg_coarse_iters, op64_, scr, r32_.as<float>(),
                                                       r_.as<double>(), tma));
        else
            throw Error(MF3D_E_INVALID, "unknown precision");
        bytes_ += vc_->bytes();
        z_.alloc(n * vc_->z_elt());
        bytes_ += z_.bytes;
        flexible_ = cfg.flexible < 0 ? (prec != MF3D_PREC_FP64) : (cfg.flexible != 0);
        host_state_ = nullptr;
        MF3D_CK(cudaMallocHost(&host_state_, sizeof(PcgState)));
        MF3D_CK(cudaEventCreate(&ev0_));
        MF3D_CK(cudaEventCreate(&ev1_));
        MF3D_CK(cudaStreamSynchronize(stream_));
    }

    ~HeadSolver() {
        if (loop_exec_) cudaGraphExecDestroy(loop_exec_);
        if (loop_graph_) cudaGraphDestroy(loop_graph_);
        if (host_state_) cudaFreeHost(host_state_);
        if (ev0_) cudaEventDestroy(ev0_);
        if (ev1_) cudaEventDestroy(ev1_);
        if (own_stream_) {
            cudaStreamSynchronize(own_stream_);
            cudaStreamDestroy(own_stream_);
        }
    }

    int num_levels() const { return (int)G_.size(); }
    long long device_bytes() const { return (long long)bytes_; }
    void coarse_info(int* first, int* ctas) const {
        if (first) *first = cplan_.Lc >= 0 ? cplan_.Lc : Lt_;
        if (ctas) *ctas = cplan_.Lc >= 0 ? cplan_.cn : 0;
    }

    void set_K(const double* K) {
        if (!K) throw Error(MF3D_E_INVALID, "K is null");
        const long long l0 = g_launches;
        cudaStream_t s = stream_;
        const int nl = (int)G_.size();
        MF3D_CK(cudaMemcpyAsync(Klev_[0]->p, K, G_[0].n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        for (int l = 0; l + 1 < nl; ++l) {
            const Geom& c = G_[l + 1];
            const ColLaunch cl = col_launch(c.nx, c.ny, c.nz);
            coarsen_kernel<<<cl.grid, cl.block, 0, s>>>(c.nx, c.ny, c.nz, Klev_[l]->as<double>(),
                                                        Klev_[l + 1]->as<double>(), cl.zchunk);
            MF3D_LAUNCH_CK();
        }
        std::vector<const double*> Kp(nl);
        for (int l = 0; l < nl; ++l) Kp[l] = Klev_[l]->as<double>();
        for (int l = 0; l < nl; ++l)
            if (coef64_[l]) launch_faces<double>(s, G_[l], Kp[l], bc_, 1.0, op64_[l]);
        vc_->build_coefs(s, Kp);
        {
            const ColLaunch cl = col_launch(G_[0].nx, G_[0].ny, G_[0].nz);
            rhs_guess_kernel<<<cl.grid, cl.block, 0, s>>>(G_[0].nx, G_[0].ny, G_[0].nz, G_[0].dx, Kp[0], to_dev(bc_),
                                                          b_.as<double>(), x0_.as<double>(), cl.zchunk);
        }
        MF3D_LAUNCH_CK();
        setup_launches_ = (int)(g_launches - l0);
        have_K_ = true;
    }

    int setup_launches() const { return setup_launches_; }
    void set_budget_ns(unsigned long long ns) { budget_ns_ = ns; }

    void vcycle(const double* r, double* z) {
        if (!have_K_) throw Error(MF3D_E_STATE, "set_K must be called before vcycle");
        const size_t n = G_[0].n;
        MF3D_CK(cudaMemcpyAsync(r_.p, r, n * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
        if (r32_.p) {
            convert_kernel<float, double><<<grid1d(n, 256), 256, 0, stream_>>>(n, r_.as<double>(), r32_.as<float>());
            MF3D_LAUNCH_CK();
        }
        if (vc_->z_elt() == sizeof(double)) {
            vc_->run(stream_, z, nullptr);
        } else {
            vc_->run(stream_, z_.p, nullptr);
            convert_kernel<double, float><<<grid1d(n, 256), 256, 0, stream_>>>(n, z_.as<float>(), z);
            MF3D_LAUNCH_CK();
        }
        MF3D_CK(cudaStreamSynchronize(stream_));
        check_err();
    }

    void check_err() {
        int e = 0;
        MF3D_CK(cudaMemcpy(&e, err_.p, sizeof(int), cudaMemcpyDeviceToHost));
        if (e) {
            MF3D_CK(cudaMemset(err_.p, 0, sizeof(int)));
            throw Error(MF3D_E_CUDA, "a TMA pipeline wait timed out in the smoother");
        }
    }

    void solve(double* h, const double* x0, mf3d_solve_result* res) {
        if (!have_K_) throw Error(MF3D_E_STATE, "set_K must be called before solve");
        if (!h) throw Error(MF3D_E_INVALID, "h is null");
        cudaStream_t s = stream_;
        const size_t n = G_[0].n;
        const long long l0 = g_launches;
        long long body_runs = 0;
        MF3D_CK(cudaEventRecord(ev0_, s));
        MF3D_CK(cudaMemcpyAsync(x_.p, x0 ? x0 : x0_.p, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        MF3D_CK(cudaMemsetAsync(tickets_.p, 0, tickets_.bytes, s));
        const bool mg = cfg_.solver == MF3D_SOLVER_MG, cg = cfg_.solver == MF3D_SOLVER_CG;
        pcg_init_kernel<<<1, 1, 0, s>>>(state_.as<PcgState>(), mg ? cfg_.mg_max_cycles : cfg_.cg_max_iter,
                                        mg ? 1 : cfg_.cg_check_every, (flexible_ && !cg) ? 1 : 0,
                                        mg ? cfg_.rtol : cfg_.cg_rtol, budget_ns_, cfg_.solver);
        MF3D_LAUNCH_CK();
        launch_residual(s, 0);
        if (cfg_.use_graph) {
            if (!loop_exec_) build_loop_graph();
            MF3D_CK(cudaGraphLaunch(loop_exec_, s));
            body_runs = -1; // known once the iteration count is back
        } else {
            // host-driven loop: one iteration per launch sequence, stop flag polled each time
            const int cap = cfg_.solver == MF3D_SOLVER_MG ? cfg_.mg_max_cycles : cfg_.cg_max_iter;
            for (int it = 0; it < std::max(cap, 1); ++it) {
                record_body(s, false);
                ++body_runs;
                MF3D_CK(cudaMemcpyAsync(host_state_, state_.p, sizeof(PcgState), cudaMemcpyDeviceToHost, s));
                MF3D_CK(cudaStreamSynchronize(s));
                if (host_state_->stop) break;
            }
        }
        launch_residual(s, 1);
        MF3D_CK(cudaMemcpyAsync(h, x_.p, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        MF3D_CK(cudaEventRecord(ev1_, s));
        MF3D_CK(cudaMemcpyAsync(host_state_, state_.p, sizeof(PcgState), cudaMemcpyDeviceToHost, s));
        MF3D_CK(cudaStreamSynchronize(s));
        check_err();
        const PcgState& st = *host_state_;
        long long launches = g_launches - l0;
        if (body_runs < 0) launches += (long long)std::max(st.iter, 1) * body_launches_;
        if (res) {
            std::memset(res, 0, sizeof(*res));
            res->num_iterations = st.iter;
            res->converged = st.converged;
            res->status = st.status;
            res->num_levels = (int)G_.size();
            res->initial_residual = std::sqrt(st.r0sq);
            res->final_residual = st.final_res;
            res->b_norm = std::sqrt(st.bb);
            res->true_rel_residual = st.bb > 0 ? std::sqrt(st.rr_true / st.bb) : std::sqrt(st.rr_true);
            float ms = 0.f;
            MF3D_CK(cudaEventElapsedTime(&ms, ev0_, ev1_));
            res->device_ms = ms;
            res->kernel_launches = (int)launches;
        }
    }

    // Times each kernel of one PCG iteration on the current state (see mf3d.h).
    std::vector<mf3d_kernel_timing> profile(int reps) {
        if (!have_K_) throw Error(MF3D_E_STATE, "set_K must be called before profile");
        reps = std::min(reps, std::max(1, cfg_.cg_max_iter - 2)); // stays inside the loop bound
        Timer tm{ev0_, ev1_, stream_};
        std::vector<mf3d_kernel_timing> out;
        const size_t n = G_[0].n;
        PcgState* st = state_.as<PcgState>();
        const double nd = (double)n, ez = (double)vc_->z_elt();
        vc_->profile(tm, reps, z_.p, &st->rho_new, out);
        const unsigned nb = grid1d(n, PK_NT);
        pcg_reopen_kernel<<<1, 1, 0, stream_>>>(st);
        MF3D_LAUNCH_CK();
        out.push_back(timing("pupdate_matvec_dot", tm.mean_ms(reps, [&] { launch_pmatvec(stream_); }),
                             (48.0 + ez) * nd, 1));
        out.push_back(timing("residual_true", tm.mean_ms(reps, [&] { launch_residual(stream_, 1); }), 48.0 * nd, 0));
        out.push_back(timing("xr_update", tm.mean_ms(reps, [&] {
            if (vc_->z_elt() == sizeof(double))
                xr_update_kernel<double><<<nb, PK_NT, 0, stream_>>>(n, x_.as<double>(), p_.as<double>(), r_.as<double>(),
                                                                   Ap_.as<double>(), z_.as<double>(), st,
                                                                   partials_.as<double>(), tickets_.as<unsigned>() + 4,
                                                                   cond_, 0, r32_.as<float>(), p2_.as<double>());
            else
                xr_update_kernel<float><<<nb, PK_NT, 0, stream_>>>(n, x_.as<double>(), p_.as<double>(), r_.as<double>(),
                                                                  Ap_.as<double>(), z_.as<float>(), st,
                                                                  partials_.as<double>(), tickets_.as<unsigned>() + 4,
                                                                  cond_, 0, r32_.as<float>(), p2_.as<double>());
            MF3D_LAUNCH_CK();
        }), 48.0 * nd + (flexible_ ? ez * nd : 0.0), 1));
        return out;
    }

    cudaStream_t stream() const { return stream_; }

  private:
    unsigned long long budget_ns_ = kSolveBudgetNs;
    // p = z + beta p fused with Ap = A p and <p, Ap> (z = r for plain CG)
    void launch_pmatvec(cudaStream_t s) {
        PcgState* st = state_.as<PcgState>();
        const ColLaunch cl = col_launch(G_[0].nx, G_[0].ny, G_[0].nz, MF3D_PMATVEC_PERSM);
        const bool z64 = cfg_.solver == MF3D_SOLVER_CG || vc_->z_elt() == sizeof(double);
        // per call: the attribute belongs to the current device
        if (z64)
            MF3D_CK(cudaFuncSetAttribute(pmatvec_dot_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)pmv_smem_bytes<double>()));
        else
            MF3D_CK(cudaFuncSetAttribute(pmatvec_dot_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)pmv_smem_bytes<float>()));
        if (z64) {
            const double* z = cfg_.solver == MF3D_SOLVER_CG ? r_.as<double>() : z_.as<double>();
            pmatvec_dot_kernel<double><<<cl.grid, cl.block, pmv_smem_bytes<double>(), s>>>(
                op64_[0], z, p_.as<double>(), p2_.as<double>(), Ap_.as<double>(), st, partials_.as<double>(),
                tickets_.as<unsigned>() + 3, cl.zchunk);
        } else {
            pmatvec_dot_kernel<float><<<cl.grid, cl.block, pmv_smem_bytes<float>(), s>>>(
                op64_[0], z_.as<float>(), p_.as<double>(), p2_.as<double>(), Ap_.as<double>(), st,
                partials_.as<double>(), tickets_.as<unsigned>() + 3, cl.zchunk);
        }
        MF3D_LAUNCH_CK();
    }

    void launch_residual(cudaStream_t s, int mode) {
        const size_t n = G_[0].n;
        double* out = mode == 0 ? r_.as<double>() : Ap_.as<double>();
        (void)n;
        const ColLaunch cl = col_launch(G_[0].nx, G_[0].ny, G_[0].nz);
        residual_kernel<double><<<cl.grid, cl.block, 0, s>>>(
            op64_[0], x_.as<double>(), b_.as<double>(), out, state_.as<PcgState>(), partials_.as<double>(),
            tickets_.as<unsigned>() + 2, mode, cfg_.conv_norm == MF3D_CONV_B ? 1 : 0,
            mode == 1 ? nullptr : r32_.as<float>(), cond_, 0, cl.zchunk);
        MF3D_LAUNCH_CK();
    }

    // One iteration (loop body) of the configured solver.
    void record_body(cudaStream_t s, bool with_cond) {
        const size_t n = G_[0].n;
        PcgState* st = state_.as<PcgState>();
        const unsigned nb = grid1d(n, PK_NT);
        const bool z64 = vc_->z_elt() == sizeof(double);
        if (cfg_.solver == MF3D_SOLVER_MG) {
            // v_cycle_recursive on (x, b) = x + V-cycle(b - A x) for the affine smoother
            vc_->run(s, z_.p, nullptr);
            if (z64) mg_xupdate_kernel<double><<<nb, PK_NT, 0, s>>>(n, x_.as<double>(), z_.as<double>(), st);
            else mg_xupdate_kernel<float><<<nb, PK_NT, 0, s>>>(n, x_.as<double>(), z_.as<float>(), st);
            MF3D_LAUNCH_CK();
            const ColLaunch cl = col_launch(G_[0].nx, G_[0].ny, G_[0].nz);
            residual_kernel<double><<<cl.grid, cl.block, 0, s>>>(op64_[0], x_.as<double>(), b_.as<double>(),
                                                                 r_.as<double>(), st, partials_.as<double>(),
                                                                 tickets_.as<unsigned>() + 2, 2,
                                                                 cfg_.conv_norm == MF3D_CONV_B ? 1 : 0,
                                                                 r32_.as<float>(), cond_, with_cond ? 1 : 0, cl.zchunk);
            MF3D_LAUNCH_CK();
            return;
        }
        const bool cg = cfg_.solver == MF3D_SOLVER_CG;
        if (!cg) vc_->run(s, z_.p, &st->rho_new);
        launch_pmatvec(s);
        if (cg || z64) {
            const double* z = cg ? r_.as<double>() : z_.as<double>();
            xr_update_kernel<double><<<nb, PK_NT, 0, s>>>(n, x_.as<double>(), p_.as<double>(), r_.as<double>(),
                                                          Ap_.as<double>(), z, st, partials_.as<double>(),
                                                          tickets_.as<unsigned>() + 4, cond_, with_cond ? 1 : 0,
                                                          r32_.as<float>(), p2_.as<double>());
        } else {
            xr_update_kernel<float><<<nb, PK_NT, 0, s>>>(n, x_.as<double>(), p_.as<double>(), r_.as<double>(),
                                                         Ap_.as<double>(), z_.as<float>(), st, partials_.as<double>(),
                                                         tickets_.as<unsigned>() + 4, cond_, with_cond ? 1 : 0,
                                                         r32_.as<float>(), p2_.as<double>());
        }
        MF3D_LAUNCH_CK();
    }

    void build_loop_graph() {
        MF3D_CK(cudaGraphCreate(&loop_graph_, 0));
        MF3D_CK(cudaGraphConditionalHandleCreate(&cond_, loop_graph_, 1u, cudaGraphCondAssignDefault));
        cudaGraphNodeParams cp{};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = cond_;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        MF3D_CK(cudaGraphAddNode(&node, loop_graph_, nullptr, 0, &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        cudaStream_t cs;
        MF3D_CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        MF3D_CK(cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        const long long l0 = g_launches;
        try {
            record_body(cs, true);
            body_launches_ = (int)(g_launches - l0);
            g_launches = l0; // captured, not launched
        } catch (...) {
            cudaGraph_t tmp;
            cudaStreamEndCapture(cs, &tmp);
            cudaStreamDestroy(cs);
            throw;
        }
        cudaGraph_t tmp;
        MF3D_CK(cudaStreamEndCapture(cs, &tmp));
        MF3D_CK(cudaStreamDestroy(cs));
        MF3D_CK(cudaGraphInstantiate(&loop_exec_, loop_graph_, 0));
    }

    mf3d_grid grid_;
    mf3d_bc bc_;
    mf3d_solver_config cfg_;
    bool pin_ = false;
    bool flexible_ = false;
    bool have_K_ = false;
    std::vector<Geom> G_;
    int Lt_ = 0;
    CoarsePlan cplan_;
    cudaStream_t stream_ = nullptr, own_stream_ = nullptr;
    std::vector<LevelOp<double>> op64_;
    std::vector<std::unique_ptr<CoefStore>> coef64_;
    std::vector<std::unique_ptr<DevMem>> Klev_;
    DevMem x_, b_, r_, p_, p2_, Ap_, x0_, z_; // p_, p2_: search directions, alternating by iteration
    DevMem partials_, tickets_, state_, mb_, err_, r32_;
    std::unique_ptr<VCycleBase> vc_;
    PcgState* host_state_ = nullptr;
    cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
    cudaGraph_t loop_graph_ = nullptr;
    cudaGraphExec_t loop_exec_ = nullptr;
    cudaGraphConditionalHandle cond_ = 0;
    size_t bytes_ = 0;
    int setup_launches_ = 0, body_launches_ = 0;
};

// ---------------------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3",
// SC'11), used for the K-field modes: counter = (mode, draw, 0, 0), key = seed.
// ---------------------------------------------------------------------------------------
struct Philox {
    static void round(uint32_t c[4], uint32_t k[2]) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        const uint32_t n0 = hi1 ^ c[1] ^ k[0], n1 = lo1, n2 = hi0 ^ c[3] ^ k[1], n3 = lo0;
        c[0] = n0;
        c[1] = n1;
        c[2] = n2;
        c[3] = n3;
        k[0] += 0x9E3779B9u;
        k[1] += 0xBB67AE85u;
    }
    static void gen(uint64_t seed, uint32_t c0, uint32_t c1, uint32_t out[4]) {
        uint32_t c[4] = {c0, c1, 0u, 0u};
        uint32_t k[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
        for (int r = 0; r < 10; ++r) round(c, k);
        for (int q = 0; q < 4; ++q) out[q] = c[q];
    }
};

// uniform double in (0,1) from 64 random bits
static double u01(uint32_t a, uint32_t b) {
    const uint64_t v = ((uint64_t)(a >> 5) << 26) | (uint64_t)(b >> 6); // 53 bits
    return ((double)v + 0.5) / 9007199254740992.0;
}

struct ModeRng {
    uint64_t seed;
    uint32_t mode, draw = 0;
    uint32_t buf[4];
    int have = 0;
    double next() {
        if (have == 0) {
            Philox::gen(seed, mode, draw++, buf);
            have = 2;
        }
        const double u = have == 2 ? u01(buf[0], buf[1]) : u01(buf[2], buf[3]);
        --have;
        return u;
    }
};

} // namespace mf3d

// =========================================================================================
// C-ABI
// =========================================================================================
using namespace mf3d;

struct mf3d_head_solver {
    std::unique_ptr<HeadSolver> impl;
};

template <class F> static int guard(F&& f) {
    try {
        f();
        return MF3D_OK;
    } catch (const Error& e) {
        g_err = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        g_err = "host allocation failed";
        return MF3D_E_NOMEM;
    } catch (const std::exception& e) {
        g_err = e.what();
        return MF3D_E_INVALID;
    }
}

static void need(const void* p, const char* what) {
    if (!p) throw Error(MF3D_E_INVALID, std::string(what) + " is null");
}

static void check_grid(const mf3d_grid* g) {
    need(g, "grid");
    if (g->nx < 1 || g->ny < 1 || g->nz < 1) throw Error(MF3D_E_INVALID, "grid sizes must be positive");
    if (!(g->dx > 0)) throw Error(MF3D_E_INVALID, "dx must be positive");
    if ((double)g->nx * g->ny * g->nz > 2147483647.0)
        throw Error(MF3D_E_INVALID, "grid exceeds 2^31 cells");
}

extern "C" {

const char* mf3d_last_error(void) { return g_err.c_str(); }
const char* mf3d_version(void) { return "mf3d-b200 0.1 (sm_100a)"; }

int mf3d_default_config(mf3d_solver_config* c) {
    return guard([&] {
        need(c, "cfg");
        std::memset(c, 0, sizeof(*c));
        c->solver = MF3D_SOLVER_PCG_MG;
        c->mg_levels = 4;
        c->mg_pre_smooth = 2;
        c->mg_post_smooth = 2;
        c->mg_max_cycles = 20;
        c->mg_coarse_iters = 50;
        c->cg_max_iter = 1000;
        c->cg_check_every = 10;
        c->cg_rtol = 1e-8;
        c->rtol = 1e-6;
        c->pin_mode = MF3D_PIN_AUTO;
        c->precision = MF3D_PREC_FP64;
        c->flexible = -1;
        c->conv_norm = MF3D_CONV_R0;
        c->use_graph = 1;
    });
}

int mf3d_head_solver_create(const mf3d_grid* grid, const mf3d_bc* bc, const mf3d_solver_config* cfg, void* stream,
                            mf3d_head_solver** out) {
    return guard([&] {
        check_grid(grid);
        need(bc, "bc");
        need(cfg, "cfg");
        need(out, "out");
        *out = nullptr;
        std::unique_ptr<mf3d_head_solver> s(new mf3d_head_solver());
        s->impl.reset(new HeadSolver(*grid, *bc, *cfg, (cudaStream_t)stream));
        *out = s.release();
    });
}

int mf3d_head_solver_destroy(mf3d_head_solver* s) {
    return guard([&] { delete s; });
}

int mf3d_head_solver_num_levels(const mf3d_head_solver* s) { return s ? s->impl->num_levels() : MF3D_E_INVALID; }

long long mf3d_head_solver_device_bytes(const mf3d_head_solver* s) { return s ? s->impl->device_bytes() : -1; }

int mf3d_head_solver_coarse_info(const mf3d_head_solver* s, int* first_level, int* cluster_ctas) {
    if (!s) return MF3D_E_INVALID;
    s->impl->coarse_info(first_level, cluster_ctas);
    return MF3D_OK;
}

int mf3d_head_solver_set_K(mf3d_head_solver* s, const double* K) {
    return guard([&] {
        need(s, "solver");
        s->impl->set_K(K);
    });
}

int mf3d_head_solve(mf3d_head_solver* s, double* h, const double* x0, mf3d_solve_result* res) {
    return guard([&] {
        need(s, "solver");
        s->impl->solve(h, x0, res);
    });
}

int mf3d_head_solver_setup_launches(const mf3d_head_solver* s) {
    return s ? s->impl->setup_launches() : MF3D_E_INVALID;
}

int mf3d_head_solver_set_time_budget(mf3d_head_solver* s, double seconds) {
    return guard([&] {
        need(s, "solver");
        if (!(seconds > 0.0) || seconds > 1e6) throw Error(MF3D_E_INVALID, "time budget must be in (0, 1e6] seconds");
        s->impl->set_budget_ns((unsigned long long)(seconds * 1e9));
    });
}

// Bounded-wait self-test: an mbarrier whose phase nothing completes (arrive = 0) or that one
// arrival completes (arrive = 1), waited on by one thread with `tries` polls of the smoother's
// wait (which = 0) or the convolution's (which = 1).  No copy is in flight: giving up leaves
// nothing behind.
__global__ void bounded_wait_kernel(int which, int arrive, int tries, int* out) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x != 0) return;
    mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    if (arrive) mbar_arrive(&bar);
    const bool ok = which == 0 ? mbar_wait(&bar, 0u, tries) : nn::nn_mbar_wait(&bar, 0u, tries);
    out[0] = ok ? 0 : 1;
}

int mf3d_diag_bounded_wait(int which, int arrive, int tries, int* gave_up_host) {
    return guard([&] {
        need(gave_up_host, "gave_up_host");
        if ((which != 0 && which != 1) || tries < 1 || tries > (1 << 22))
            throw Error(MF3D_E_INVALID, "which must be 0 or 1, tries in [1, 2^22]");
        DevMem out(sizeof(int));
        MF3D_CK(cudaMemset(out.p, 0xff, sizeof(int)));
        bounded_wait_kernel<<<1, 32>>>(which, arrive ? 1 : 0, tries, out.as<int>());
        MF3D_LAUNCH_CK();
        MF3D_CK(cudaMemcpy(gave_up_host, out.p, sizeof(int), cudaMemcpyDeviceToHost));
    });
}

int mf3d_head_solver_profile(mf3d_head_solver* s, int reps, mf3d_kernel_timing* out, int cap, int* count) {
    return guard([&] {
        need(s, "solver");
        need(out, "out");
        need(count, "count");
        auto v = s->impl->profile(std::max(1, reps));
        *count = (int)std::min<size_t>(v.size(), (size_t)std::max(cap, 0));
        for (int i = 0; i < *count; ++i) out[i] = v[i];
    });
}

int mf3d_head_solver_vcycle(mf3d_head_solver* s, const double* r, double* z) {
    return guard([&] {
        need(s, "solver");
        need(r, "r");
        need(z, "z");
        s->impl->vcycle(r, z);
    });
}

static void run_velocity(const mf3d_grid* g, const mf3d_bc* bc, const double* h, const double* K, int layout,
                         double* U, double* V, double* W, double* out_host, cudaStream_t s) {
    check_grid(g);
    need(bc, "bc");
    validate_bc(*bc);
    need(h, "h");
    need(K, "K");
    need(U, "U");
    need(V, "V");
    need(W, "W");
    if (layout != MF3D_VEL_COMPACT && layout != MF3D_VEL_PADDED) throw Error(MF3D_E_INVALID, "unknown layout");
    const size_t n = (size_t)g->nx * g->ny * g->nz;
    VelOut o{U, V, W, layout};
    if (!out_host) {
        const ColLaunch cl = col_launch(g->nx, g->ny, g->nz);
        velocity_kernel<<<cl.grid, cl.block, 0, s>>>(g->nx, g->ny, g->nz, g->dx, h, K, to_dev(*bc), o, nullptr, nullptr,
                                                     nullptr, nullptr, cl.zchunk);
        MF3D_LAUNCH_CK();
        return;
    }
    const ColLaunch cl = col_launch(g->nx, g->ny, g->nz);
    const unsigned nb = cl.nblocks;
    DevMem scratch((size_t)nb * 2 * sizeof(double) + 64);
    char* base = scratch.as<char>();
    unsigned long long* mx = (unsigned long long*)base;
    unsigned* ticket = (unsigned*)(base + 8);
    double* sums = (double*)(base + 16);
    double* partials = (double*)(base + 64);
    MF3D_CK(cudaMemsetAsync(base, 0, 64, s));
    velocity_kernel<<<cl.grid, cl.block, 0, s>>>(g->nx, g->ny, g->nz, g->dx, h, K, to_dev(*bc), o, mx, partials, ticket,
                                                 sums, cl.zchunk);
    MF3D_LAUNCH_CK();
    unsigned long long hb[4];
    MF3D_CK(cudaMemcpyAsync(hb, base, 32, cudaMemcpyDeviceToHost, s));
    MF3D_CK(cudaStreamSynchronize(s));
    double d[3];
    std::memcpy(&d[0], &hb[0], 8);
    std::memcpy(&d[1], &hb[2], 8);
    std::memcpy(&d[2], &hb[3], 8);
    out_host[0] = d[0];
    out_host[1] = d[1];
    out_host[2] = d[2];
}

int mf3d_velocity_from_head(const mf3d_grid* g, const mf3d_bc* bc, const double* h, const double* K, int layout,
                            double* U, double* V, double* W, void* stream) {
    return guard([&] { run_velocity(g, bc, h, K, layout, U, V, W, nullptr, (cudaStream_t)stream); });
}

int mf3d_velocity_mass_balance(const mf3d_grid* g, const mf3d_bc* bc, const double* h, const double* K, double* U,
                               double* V, double* W, double* out_host, void* stream) {
    return guard([&] {
        need(out_host, "out_host");
        run_velocity(g, bc, h, K, MF3D_VEL_COMPACT, U, V, W, out_host, (cudaStream_t)stream);
    });
}

int mf3d_velocity_diagnostics(const mf3d_grid* g, int layout, const double* U, const double* V, const double* W,
                              double* div, double* omag, double* hel, double* stats_host, void* stream) {
    return guard([&] {
        check_grid(g);
        need(U, "U");
        need(V, "V");
        need(W, "W");
        if (layout != MF3D_VEL_COMPACT && layout != MF3D_VEL_PADDED) throw Error(MF3D_E_INVALID, "unknown layout");
        cudaStream_t s = (cudaStream_t)stream;
        const ColLaunch cl = col_launch(g->nx, g->ny, g->nz);
        // temporary reduction scratch, as the reference's compute_field_stats allocates its own
        DevMem scr(stats_host ? (9 * (size_t)cl.nblocks + 16) * sizeof(double) : 0);
        double* partials = stats_host ? scr.as<double>() : nullptr;
        double* stats_dev = stats_host ? partials + 9 * (size_t)cl.nblocks : nullptr;
        unsigned* ticket = stats_host ? reinterpret_cast<unsigned*>(stats_dev + 9) : nullptr;
        if (stats_host) MF3D_CK(cudaMemsetAsync(ticket, 0, sizeof(unsigned), s));
        velocity_diag_kernel<<<cl.grid, cl.block, 0, s>>>(g->nx, g->ny, g->nz, 1.0 / g->dx, layout, U, V, W, div,
                                                          omag, hel, partials, ticket, stats_dev, cl.zchunk);
        MF3D_LAUNCH_CK();
        if (stats_host) MF3D_CK(cudaMemcpyAsync(stats_host, stats_dev, 9 * sizeof(double), cudaMemcpyDeviceToHost, s));
        MF3D_CK(cudaStreamSynchronize(s));
    });
}

// ---- mass balance with static scratch (no device allocation) -------------------------------
// The reduction scratch of the fused velocity + mass-balance kernel (max bits, ticket, two
// sums, then two partial sums per block) lives in one file-scope device array, so this entry
// point calls neither cudaMalloc nor cudaFree.  One array exists per device: calls that
// overlap on the same device (two streams or two host threads) share it and race.
namespace {
constexpr unsigned kMbNoAllocMaxBlocks = MF3D_MB_NOALLOC_MAX_BLOCKS;
constexpr size_t kMbNoAllocHeader = 64;
constexpr size_t kMbNoAllocBytes = kMbNoAllocHeader + (size_t)kMbNoAllocMaxBlocks * 2 * sizeof(double);
static __device__ __align__(256) unsigned char g_mb_scratch[kMbNoAllocBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mb_mu;
unsigned char* g_mb_ptr[kMaxDevices] = {};

// Device address of g_mb_scratch on the current device, looked up once per device with that
// device current.  The first call on a device does the lookup (which may load the module on
// that device), so on each device that first call should come before any stream capture.
unsigned char* mb_scratch_on_current_device() {
    int dev = 0;
    MF3D_CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) throw Error(MF3D_E_INVALID, "device ordinal out of range for static scratch");
    std::lock_guard<std::mutex> lock(g_mb_mu);
    if (!g_mb_ptr[dev]) {
        unsigned char* ptr = nullptr;
        const cudaError_t e = cudaGetSymbolAddress((void**)&ptr, g_mb_scratch);
        if (e != cudaSuccess || !ptr)
            throw Error(MF3D_E_CUDA, std::string("cudaGetSymbolAddress(static scratch) failed: ") + cudaGetErrorString(e));
        g_mb_ptr[dev] = ptr;
    }
    return g_mb_ptr[dev];
}
} // namespace

int mf3d_velocity_mass_balance_noalloc(const mf3d_grid* g, const mf3d_bc* bc, const double* h, const double* K,
                                       double* U, double* V, double* W, double* out_host, void* stream) {
    return guard([&] {
        check_grid(g);
        need(bc, "bc");
        validate_bc(*bc);
        need(h, "h");
        need(K, "K");
        need(U, "U");
        need(V, "V");
        need(W, "W");
        need(out_host, "out_host");
        cudaStream_t s = (cudaStream_t)stream;
        const ColLaunch cl = col_launch(g->nx, g->ny, g->nz);
        if (cl.nblocks > kMbNoAllocMaxBlocks)
            throw Error(MF3D_E_INVALID, "grid too large for the static mass-balance scratch: " + std::to_string(cl.nblocks) +
                                            " reduction blocks needed, at most " +
                                            std::to_string(kMbNoAllocMaxBlocks) +
                                            " (ceil(nx/32) * ceil(ny/8) must not exceed it)");
        unsigned char* base = mb_scratch_on_current_device();
        unsigned long long* mx = (unsigned long long*)base;
        unsigned* ticket = (unsigned*)(base + 8);
        double* sums = (double*)(base + 16);
        double* partials = (double*)(base + kMbNoAllocHeader);
        // max bits, ticket and sums must start at zero; the partials are written before read
        MF3D_CK(cudaMemsetAsync(base, 0, kMbNoAllocHeader, s));
        VelOut o{U, V, W, MF3D_VEL_COMPACT};
        velocity_kernel<<<cl.grid, cl.block, 0, s>>>(g->nx, g->ny, g->nz, g->dx, h, K, to_dev(*bc), o, mx, partials,
                                                     ticket, sums, cl.zchunk);
        MF3D_LAUNCH_CK();
        unsigned long long hb[4];
        MF3D_CK(cudaMemcpyAsync(hb, base, 32, cudaMemcpyDeviceToHost, s));
        MF3D_CK(cudaStreamSynchronize(s));
        std::memcpy(&out_host[0], &hb[0], 8);
        std::memcpy(&out_host[1], &hb[2], 8);
        std::memcpy(&out_host[2], &hb[3], 8);
    });
}

// ---- operator pieces ----------------------------------------------------------------------
struct OneLevel {
    Geom G;
    CoefStore cs;
    LevelOp<double> op;
    OneLevel(const mf3d_grid* g, const mf3d_bc* bc, int pin, const double* K, cudaStream_t s) {
        check_grid(g);
        need(bc, "bc");
        validate_bc(*bc);
        need(K, "K");
        G = Geom{g->nx, g->ny, g->nz, (size_t)g->nx * g->ny * g->nz, g->dx};
        op = make_op<double>(G, *bc, pin != 0, 1.0);
        cs.build<double>(G, sizeof(double), op);
        launch_faces<double>(s, G, K, *bc, 1.0, op);
    }
};

__global__ void apply_A_kernel(const LevelOp<double> L, const double* __restrict__ x, double* __restrict__ y) {
    const size_t n = (size_t)L.nx * L.ny * L.nz;
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(c % L.nx), j = (int)((c / L.nx) % L.ny), k = (int)(c / ((size_t)L.nx * L.ny));
        y[c] = apply_A_cell(L, x, i, j, k, c);
    }
}

// r = b - A x with the smoother's pin convention (full diagonal doubled at cell 0,
// src/multigrid/smoothers/residual_3d.cu:365-368).
__global__ void residual_mg_kernel(const LevelOp<double> L, const double* __restrict__ x, const double* __restrict__ b,
                                   double* __restrict__ r) {
    const size_t n = (size_t)L.nx * L.ny * L.nz;
    LevelOp<double> Lnp = L;
    Lnp.pin = 0;
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(c % L.nx), j = (int)((c / L.nx) % L.ny), k = (int)(c / ((size_t)L.nx * L.ny));
        double ax = apply_A_cell(Lnp, x, i, j, k, c);
        if (L.pin && c == 0) {
            double cxm, cxp, cym, cyp, czm, czp;
            cell_coefs<double>(L, i, j, k, c, cxm, cxp, cym, cyp, czm, czp);
            ax -= (cxm + cxp + cym + cyp + czm + czp) * x[c] * L.inv_dx2;
        }
        r[c] = b[c] - ax;
    }
}

int mf3d_apply_A(const mf3d_grid* g, const mf3d_bc* bc, int pin, const double* K, const double* x, double* y,
                 void* stream) {
    return guard([&] {
        cudaStream_t s = (cudaStream_t)stream;
        need(x, "x");
        need(y, "y");
        OneLevel L(g, bc, pin, K, s);
        apply_A_kernel<<<grid1d(L.G.n, 256), 256, 0, s>>>(L.op, x, y);
        MF3D_LAUNCH_CK();
        MF3D_CK(cudaStreamSynchronize(s));
    });
}

int mf3d_residual(const mf3d_grid* g, const mf3d_bc* bc, int pin, const double* K, const double* x, const double* b,
                  double* r, void* stream) {
    return guard([&] {
        cudaStream_t s = (cudaStream_t)stream;
        need(x, "x");
        need(b, "b");
        need(r, "r");
        OneLevel L(g, bc, pin, K, s);
        residual_mg_kernel<<<grid1d(L.G.n, 256), 256, 0, s>>>(L.op, x, b, r);
        MF3D_LAUNCH_CK();
        MF3D_CK(cudaStreamSynchronize(s));
    });
}

int mf3d_gsrb(const mf3d_grid* g, const mf3d_bc* bc, int pin, const double* K, const double* b, double* x, int iters,
              void* stream) {
    return guard([&] {
        cudaStream_t s = (cudaStream_t)stream;
        need(b, "b");
        need(x, "x");
        if (iters < 0) throw Error(MF3D_E_INVALID, "iters < 0");
        for (int a = 0; a < 3; ++a) {
            const int n = a == 0 ? g->nx : (a == 1 ? g->ny : g->nz);
            if (bc && bc->type[2 * a] == MF3D_BC_PERIODIC && (n & 1))
                throw Error(MF3D_E_INVALID, "red-black smoothing needs an even cell count on a periodic axis");
        }
        OneLevel L(g, bc, pin, K, s);
        if (iters == 0) return;
        DevMem tmp(L.G.n * sizeof(double));
        double* pbufs[2] = {x, tmp.as<double>()};
        // the x-pair sweep where it applies (nx even, periodic axes whole tiles), as in the V-cycle
        if (g->nx % 2 == 0 && (bc->type[0] != MF3D_BC_PERIODIC || g->nx % SP_TX == 0) &&
            (bc->type[2] != MF3D_BC_PERIODIC || g->ny % SP_TY == 0)) {
            const bool tm = sp_tma_ok<double>(L.G, *bc);
            const int occ = tm ? pair_sweep_setup<double, double, 0, true>() : pair_sweep_setup<double, double, 0, false>();
            DevMem err(sizeof(int));
            MF3D_CK(cudaMemsetAsync(err.p, 0, sizeof(int), s));
            SpArgs<double, double> a{};
            a.L = L.op;
            a.b = b;
            a.err = err.as<int>();
            const dim3 grid = pair_grid(L.G, (long long)std::max(1, occ) * num_sms(), &a.zchunk,
                                        tm ? sp_tx<double, double, true>() : sp_tx<double, double, false>());
            SpMaps maps[2] = {};
            if (tm)
                for (int q = 0; q < 2; ++q) maps[q] = make_sp_maps<double, double>(L.G, pbufs[q], b, L.op);
            int cur = 0;
            for (int it = 0; it < iters; ++it) {
                a.x_in = pbufs[cur];
                a.x_out = pbufs[cur ^ 1];
                launch_pair_sweep<double, double>(s, grid, 0, tm, maps[cur], a);
                cur ^= 1;
            }
            int e = 0;
            MF3D_CK(cudaMemcpyAsync(&e, err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
            if (cur != 0) MF3D_CK(cudaMemcpyAsync(x, pbufs[cur], L.G.n * sizeof(double), cudaMemcpyDeviceToDevice, s));
            MF3D_CK(cudaStreamSynchronize(s));
            if (e) throw Error(MF3D_E_CUDA, "a TMA staging wait timed out in the smoother");
            return;
        }
        const int gx = (g->nx + SW_TX - 1) / SW_TX, gy = (g->ny + SW_TY - 1) / SW_TY;
        const int zc = std::max(2, std::min(64, ((g->nz + 1) & ~1)));
        dim3 grid(gx, gy, (g->nz + zc - 1) / zc);
        double* bufs[2] = {x, tmp.as<double>()};
        int cur = 0;
        for (int it = 0; it < iters; ++it) {
            SweepArgs<double, double, double> a{};
            a.L = L.op;
            a.b = b;
            a.x_in = bufs[cur];
            a.x_out = bufs[cur ^ 1];
            a.zchunk = zc;
            sweep_kernel<double, double, double, 0><<<grid, SW_NT, 0, s>>>(a);
            MF3D_LAUNCH_CK();
            cur ^= 1;
        }
        if (cur != 0) MF3D_CK(cudaMemcpyAsync(x, bufs[cur], L.G.n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        MF3D_CK(cudaStreamSynchronize(s));
    });
}

int mf3d_restrict(const mf3d_grid* c, const double* rf, double* bc_out, void* stream) {
    return guard([&] {
        check_grid(c);
        need(rf, "r_fine");
        need(bc_out, "b_coarse");
        cudaStream_t s = (cudaStream_t)stream;
        const size_t n = (size_t)c->nx * c->ny * c->nz;
        restrict_kernel<double, double><<<grid1d(n, 256), 256, 0, s>>>(c->nx, c->ny, c->nz, rf, bc_out);
        MF3D_LAUNCH_CK();
        MF3D_CK(cudaStreamSynchronize(s));
    });
}

int mf3d_prolong_add(const mf3d_grid* c, const double* xc, double* xf, void* stream) {
    return guard([&] {
        check_grid(c);
        need(xc, "x_coarse");
        need(xf, "x_fine");
        cudaStream_t s = (cudaStream_t)stream;
        const size_t nf = (size_t)8 * c->nx * c->ny * c->nz;
        prolong_kernel<double><<<grid1d(nf, 256), 256, 0, s>>>(2 * c->nx, 2 * c->ny, 2 * c->nz, xf, xc, xf);
        MF3D_LAUNCH_CK();
        MF3D_CK(cudaStreamSynchronize(s));
    });
}

int mf3d_coarsen_K(const mf3d_grid* c, const double* Kf, double* Kc, void* stream) {
    return guard([&] {
        check_grid(c);
        need(Kf, "K_fine");
        need(Kc, "K_coarse");
        cudaStream_t s = (cudaStream_t)stream;
        const size_t n = (size_t)c->nx * c->ny * c->nz;
        (void)n;
        const ColLaunch cl = col_launch(c->nx, c->ny, c->nz);
        coarsen_kernel<<<cl.grid, cl.block, 0, s>>>(c->nx, c->ny, c->nz, Kf, Kc, cl.zchunk);
        MF3D_LAUNCH_CK();
        MF3D_CK(cudaStreamSynchronize(s));
    });
}

int mf3d_build_rhs(const mf3d_grid* g, const mf3d_bc* bc, const double* K, double* b, void* stream) {
    return guard([&] {
        check_grid(g);
        need(bc, "bc");
        need(K, "K");
        need(b, "b");
        cudaStream_t s = (cudaStream_t)stream;
        const size_t n = (size_t)g->nx * g->ny * g->nz;
        (void)n;
        const ColLaunch cl = col_launch(g->nx, g->ny, g->nz);
        rhs_guess_kernel<<<cl.grid, cl.block, 0, s>>>(g->nx, g->ny, g->nz, g->dx, K, to_dev(*bc), b, nullptr, cl.zchunk);
        MF3D_LAUNCH_CK();
        MF3D_CK(cudaStreamSynchronize(s));
    });
}

__global__ void guess_kernel(int nx, int ny, int nz, BcDev bc, double* __restrict__ h) {
    const size_t n = (size_t)nx * ny * nz;
    const bool lin = bc.type[0] == BC_DIRICHLET && bc.type[1] == BC_DIRICHLET;
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(c % nx);
        h[c] = lin ? bc.value[0] + (bc.value[1] - bc.value[0]) * (((double)i + 0.5) / (double)nx) : 0.0;
    }
}

int mf3d_init_head_guess(const mf3d_grid* g, const mf3d_bc* bc, double* h, void* stream) {
    return guard([&] {
        check_grid(g);
        need(bc, "bc");
        need(h, "h");
        cudaStream_t s = (cudaStream_t)stream;
        const size_t n = (size_t)g->nx * g->ny * g->nz;
        guess_kernel<<<grid1d(n, 256), 256, 0, s>>>(g->nx, g->ny, g->nz, to_dev(*bc), h);
        MF3D_LAUNCH_CK();
        MF3D_CK(cudaStreamSynchronize(s));
    });
}

int mf3d_kfield_modes(unsigned long long seed, int n_modes, int cov, double lx, double ly, double lz,
                      double* modes) {
    return guard([&] {
        need(modes, "modes_host");
        if (n_modes <= 0) throw Error(MF3D_E_INVALID, "n_modes must be positive");
        if (!(lx > 0 && ly > 0 && lz > 0)) throw Error(MF3D_E_INVALID, "correlation lengths must be positive");
        if (cov != MF3D_COV_EXPONENTIAL && cov != MF3D_COV_GAUSSIAN) throw Error(MF3D_E_INVALID, "unknown covariance");
        const double PI = 3.14159265358979323846;
        double* k1 = modes;
        double* k2 = modes + n_modes;
        double* k3 = modes + 2 * (size_t)n_modes;
        double* a = modes + 3 * (size_t)n_modes;
        double* b = modes + 4 * (size_t)n_modes;
        for (int m = 0; m < n_modes; ++m) {
            ModeRng g{seed, (uint32_t)m};
            // direction uniform on the sphere
            const double fi = 2.0 * PI * g.next();
            const double theta = std::acos(1.0 - 2.0 * g.next());
            double k = 0.0;
            if (cov == MF3D_COV_EXPONENTIAL) {
                // radial density k^2/(1+k^2)^2 (3-D spectrum of exp(-r)): half-Cauchy proposal,
                // accept with probability k^2/(1+k^2) (stochastic.cu:70-83)
                for (int tries = 0; tries < 100000; ++tries) {
                    k = std::tan(PI * 0.5 * g.next());
                    if (g.next() < k * k / (1.0 + k * k)) break;
                }
            } else {
                // radial density k^2 exp(-k^2/2) on [0, 10] by rejection, then scaled by sqrt(2)
                // so that E cos(k.r) = exp(-r^2) (stochastic.cu:118-160)
                for (int tries = 0; tries < 100000; ++tries) {
                    k = 10.0 * g.next();
                    if (g.next() * 2.0 * std::exp(-1.0) < k * k * std::exp(-0.5 * k * k)) break;
                }
                k *= std::sqrt(2.0);
            }
            k1[m] = k * std::sin(fi) * std::sin(theta) / lx;
            k2[m] = k * std::cos(fi) * std::sin(theta) / ly;
            k3[m] = k * std::cos(theta) / lz;
            double u1 = g.next(), u2 = g.next();
            a[m] = std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * PI * u2);
            u1 = g.next();
            u2 = g.next();
            b[m] = std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * PI * u2);
        }
    });
}

int mf3d_kfield_eval(const mf3d_grid* g, int n_modes, const double* modes, double sigma2, double log_kg,
                     int want_exp, double* out, void* stream) {
    return guard([&] {
        check_grid(g);
        need(modes, "modes");
        need(out, "out");
        if (n_modes <= 0 || sigma2 < 0) throw Error(MF3D_E_INVALID, "bad n_modes or variance");
        cudaStream_t s = (cudaStream_t)stream;
        const size_t tasks = (size_t)g->ny * g->nz * ((g->nx + KF_SEG - 1) / KF_SEG);
        kfield_kernel<<<(unsigned)((tasks + KF_NT - 1) / KF_NT), KF_NT, 0, s>>>(
            g->nx, g->ny, g->nz, g->dx, n_modes, modes, std::sqrt(sigma2), log_kg, want_exp, out);
        MF3D_LAUNCH_CK();
        MF3D_CK(cudaStreamSynchronize(s));
    });
}

} // extern "C"

#include "batch.cuh"
#include "nn.cuh"
