// hea_capi.cu -- C ABI of the swap-search engine: validation, device tables,
// the search driver and the component entry points.  Declarations and the
// reference interfaces they replace: include/hea_cuda.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <chrono>
#include <ctime>
#include <deque>
#include <map>
#include <mutex>
#include <new>
#include <unordered_map>
#include <string>
#include <tuple>
#include <vector>

#include "hea_cuda.h"
#include "hea_search.cuh"
#include "hea_large.cuh"

using namespace hea;

namespace {

thread_local std::string g_error;

int fail(int code, const char *fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_error = buf;
    return code;
}

#define HEA_CUDA(call)                                                                                    \
    do {                                                                                                  \
        cudaError_t e_ = (call);                                                                          \
        if (e_ != cudaSuccess) return fail(HEA_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

// ---------------------------------------------------------------------------
// Device memory for plans, tables and the component entry points: blocks
// freed by one call are kept (per device and rounded size) and handed to the
// next call that asks for the same size, so repeated searches of one shape
// make no cudaMalloc/cudaFree (both can synchronise the device).  At most
// kPoolCacheBytes stay cached; a failed cudaMalloc releases the cache and
// retries.  Blocks go back to the cache only after the owning stream's work
// has finished (every owner synchronises before freeing).
// ---------------------------------------------------------------------------
struct DevicePool {
    std::mutex mu;
    std::map<std::pair<int, size_t>, std::vector<void *>> free_;  // (device, rounded size) -> cached blocks
    std::unordered_map<void *, std::pair<int, size_t>> live;
    size_t cached = 0;
};
// never destroyed: plans may be freed during interpreter or process shutdown
DevicePool &pool()
{
    static DevicePool *p = new DevicePool;
    return *p;
}
constexpr size_t kPoolCacheBytes = (size_t)8 << 30;

size_t pool_round(size_t b)
{
    if (b == 0) b = 1;
    if (b <= ((size_t)1 << 20)) return (b + 4095) & ~(size_t)4095;
    return (b + ((size_t)2 << 20) - 1) & ~(((size_t)2 << 20) - 1);
}

void pool_release_device(DevicePool &P, int dev)
{
    for (auto it = P.free_.begin(); it != P.free_.end();) {
        if (it->first.first != dev) {
            ++it;
            continue;
        }
        for (void *q : it->second) {
            cudaFree(q);
            P.cached -= it->first.second;
        }
        it = P.free_.erase(it);
    }
}

cudaError_t dev_alloc(void **p, size_t bytes)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const size_t r = pool_round(bytes);
    DevicePool &P = pool();
    std::lock_guard<std::mutex> lk(P.mu);
    auto it = P.free_.find({dev, r});
    if (it != P.free_.end() && !it->second.empty()) {
        *p = it->second.back();
        it->second.pop_back();
        P.cached -= r;
        P.live[*p] = {dev, r};
        return cudaSuccess;
    }
    e = cudaMalloc(p, r);
    if (e != cudaSuccess) {
        cudaGetLastError();
        pool_release_device(P, dev);
        e = cudaMalloc(p, r);
    }
    if (e == cudaSuccess) P.live[*p] = {dev, r};
    return e;
}

template <class X>
cudaError_t dev_alloc(X **p, size_t bytes)
{
    void *q = nullptr;
    const cudaError_t e = dev_alloc(&q, bytes);
    *p = static_cast<X *>(q);
    return e;
}

void dev_free(void *p)
{
    if (!p) return;
    DevicePool &P = pool();
    std::lock_guard<std::mutex> lk(P.mu);
    auto it = P.live.find(p);
    if (it == P.live.end()) {
        cudaFree(p);
        return;
    }
    const std::pair<int, size_t> key = it->second;
    P.live.erase(it);
    if (P.cached + key.second > kPoolCacheBytes) {
        cudaFree(p);
        return;
    }
    P.free_[key].push_back(p);
    P.cached += key.second;
}

#define HEA_TRY(expr)            \
    do {                         \
        int rc_ = (expr);        \
        if (rc_ != HEA_OK) return rc_; \
    } while (0)

// ---------------------------------------------------------------------------
// Kernel dispatch over (T, S)
// ---------------------------------------------------------------------------
using GenFn = void (*)(const SearchConst, const GenArgs);
using McFn = void (*)(const SearchConst, const McArgs);

#define HEA_GEN_ROW(T) {nullptr, generate_kernel<T, 1>, generate_kernel<T, 2>, generate_kernel<T, 3>}
const GenFn kGen[kMaxTypes + 1][kMaxShells + 1] = {
    {nullptr, nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr, nullptr}, HEA_GEN_ROW(2), HEA_GEN_ROW(3),
    HEA_GEN_ROW(4), HEA_GEN_ROW(5), HEA_GEN_ROW(6)};

// Local-search kernel for species count T and the table's padded shell layout:
// the layouts of the FCC/BCC shell sets (in int4 chunks per shell) have their
// loads unrolled; any other table uses the runtime-layout instance.
template <int T>
McFn pick_mc_t(int c0, int c1, int c2, int S, bool implicit)
{
    if (implicit) return S == 1 ? mc_kernel<T, ImplicitShells<1>> : S == 2 ? mc_kernel<T, ImplicitShells<2>>
                                                                          : mc_kernel<T, ImplicitShells<3>>;
    if (c0 == 2 && c1 == 0 && c2 == 0) return mc_kernel<T, Shells<2, 0, 0>>;  // BCC, 1 shell
    if (c0 == 2 && c1 == 2 && c2 == 0) return mc_kernel<T, Shells<2, 2, 0>>;  // BCC, 2 shells
    if (c0 == 2 && c1 == 2 && c2 == 3) return mc_kernel<T, Shells<2, 2, 3>>;  // BCC 8/6/12
    if (c0 == 3 && c1 == 0 && c2 == 0) return mc_kernel<T, Shells<3, 0, 0>>;  // FCC, 1 shell
    if (c0 == 3 && c1 == 2 && c2 == 0) return mc_kernel<T, Shells<3, 2, 0>>;  // FCC, 2 shells
    if (c0 == 3 && c1 == 2 && c2 == 3) return mc_kernel<T, Shells<3, 2, 3>>;  // FCC 12/6/12
    if (c0 == 3 && c1 == 2 && c2 == 6) return mc_kernel<T, Shells<3, 2, 6>>;  // FCC 12/6/24
    if (S == 1) return mc_kernel<T, RuntimeShells<1>>;
    if (S == 2) return mc_kernel<T, RuntimeShells<2>>;
    return mc_kernel<T, RuntimeShells<3>>;
}

// The same choice for the HBM-occupancy (cluster) search.
template <int T>
McFn pick_mc_large_t(int c0, int c1, int c2, int S, bool implicit)
{
    if (implicit)
        return S == 1 ? mc_large_kernel<T, ImplicitShells<1>>
                      : S == 2 ? mc_large_kernel<T, ImplicitShells<2>> : mc_large_kernel<T, ImplicitShells<3>>;
    if (c0 == 2 && c1 == 2 && c2 == 3) return mc_large_kernel<T, Shells<2, 2, 3>>;
    if (c0 == 3 && c1 == 2 && c2 == 3) return mc_large_kernel<T, Shells<3, 2, 3>>;
    if (c0 == 3 && c1 == 2 && c2 == 6) return mc_large_kernel<T, Shells<3, 2, 6>>;
    if (S == 1) return mc_large_kernel<T, RuntimeShells<1>>;
    if (S == 2) return mc_large_kernel<T, RuntimeShells<2>>;
    return mc_large_kernel<T, RuntimeShells<3>>;
}

McFn pick_mc_large(int T, int c0, int c1, int c2, int S, bool implicit)
{
    switch (T) {
    case 2: return pick_mc_large_t<2>(c0, c1, c2, S, implicit);
    case 3: return pick_mc_large_t<3>(c0, c1, c2, S, implicit);
    case 4: return pick_mc_large_t<4>(c0, c1, c2, S, implicit);
    case 5: return pick_mc_large_t<5>(c0, c1, c2, S, implicit);
    default: return pick_mc_large_t<6>(c0, c1, c2, S, implicit);
    }
}

using LGenFn = void (*)(const SearchConst, uint8_t *, const int32_t *, uint32_t);
using LRecFn = void (*)(const SearchConst, const int4 *, const uint8_t *, const int32_t *, int32_t *, uint4 *);
using LFitFn = void (*)(const SearchConst, const int32_t *, int, const int32_t *, double *);
const LGenFn kLGen[kMaxTypes + 1] = {nullptr, nullptr, large_generate_kernel<2>, large_generate_kernel<3>,
                                     large_generate_kernel<4>, large_generate_kernel<5>, large_generate_kernel<6>};
#define HEA_LREC_ROW(T) {nullptr, large_recount_kernel<T, 1>, large_recount_kernel<T, 2>, large_recount_kernel<T, 3>}
const LRecFn kLRec[kMaxTypes + 1][kMaxShells + 1] = {
    {nullptr, nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr, nullptr}, HEA_LREC_ROW(2), HEA_LREC_ROW(3),
    HEA_LREC_ROW(4), HEA_LREC_ROW(5), HEA_LREC_ROW(6)};
#define HEA_LFIT_ROW(T) {nullptr, large_fitness_kernel<T, 1>, large_fitness_kernel<T, 2>, large_fitness_kernel<T, 3>}
const LFitFn kLFit[kMaxTypes + 1][kMaxShells + 1] = {
    {nullptr, nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr, nullptr}, HEA_LFIT_ROW(2), HEA_LFIT_ROW(3),
    HEA_LFIT_ROW(4), HEA_LFIT_ROW(5), HEA_LFIT_ROW(6)};

__global__ void zero_counts_kernel(const int32_t *order, int count, int32_t *cnt, int ncount)
{
    const int p = blockIdx.y;
    if (p >= count) return;
    int32_t *g = cnt + (size_t)order[p] * ncount;
    for (int x = threadIdx.x; x < ncount; x += blockDim.x) g[x] = 0;
}

McFn pick_mc(int T, int c0, int c1, int c2, int S, bool implicit)
{
    switch (T) {
    case 2: return pick_mc_t<2>(c0, c1, c2, S, implicit);
    case 3: return pick_mc_t<3>(c0, c1, c2, S, implicit);
    case 4: return pick_mc_t<4>(c0, c1, c2, S, implicit);
    case 5: return pick_mc_t<5>(c0, c1, c2, S, implicit);
    default: return pick_mc_t<6>(c0, c1, c2, S, implicit);
    }
}

// ---------------------------------------------------------------------------
// Table preparation kernels
// ---------------------------------------------------------------------------
struct PadGeom {
    int32_t size[kMaxShells], off[kMaxShells], poff[kMaxShells], psize[kMaxShells];
    int32_t num_shells, raw_row, pad_row, num_sites;
};

// Padded copy of the raw table plus its checks: id range, no site listed as its
// own neighbour, and symmetry with multiplicity per shell (the reference's
// incremental update at accelerate.cpp:526-530 counts each pair from both
// ends, which equals a recount only on such tables).  err bits: 1 range,
// 2 self, 4 asymmetric.
__global__ void pad_and_check_kernel(const int32_t *raw, int32_t *padded, PadGeom g, int *err)
{
    const int64_t total = (int64_t)g.num_sites * g.pad_row;
    for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < total; x += (int64_t)gridDim.x * blockDim.x) {
        const int s = (int)(x / g.pad_row), e = (int)(x % g.pad_row);
        int k = 0;
        while (k + 1 < g.num_shells && e >= g.poff[k + 1]) ++k;
        const int q = e - g.poff[k];
        if (q >= g.size[k]) {
            padded[x] = g.num_sites;
            continue;
        }
        const int n = raw[(int64_t)s * g.raw_row + g.off[k] + q];
        padded[x] = n;
        if (n < 0 || n >= g.num_sites) {
            atomicOr(err, 1);
            continue;
        }
        if (n == s) {
            atomicOr(err, 2);
            continue;
        }
        // multiplicity of n in s's shell k must equal that of s in n's shell k
        const int32_t *rs = raw + (int64_t)s * g.raw_row + g.off[k];
        const int32_t *rn = raw + (int64_t)n * g.raw_row + g.off[k];
        int fwd = 0, back = 0;
        for (int j = 0; j < g.size[k]; ++j) {
            fwd += rs[j] == n;
            back += rn[j] == s;
        }
        if (fwd != back) atomicOr(err, 4);
    }
}

// Bit (n - s + N - 1) for every entry n (< N) of every site s of the padded
// table: the site-id offsets at which two sites can be neighbours.
__global__ void nbmask_kernel(const int32_t *padded, int num_sites, int pad_row, uint32_t *mask)
{
    const int64_t total = (int64_t)num_sites * pad_row;
    for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < total; x += (int64_t)gridDim.x * blockDim.x) {
        const int sidx = (int)(x / pad_row);
        const int n = padded[x];
        if (n < 0 || n >= num_sites) continue;
        const uint32_t d = (uint32_t)(n - sidx + num_sites - 1);
        atomicOr(mask + (d >> 5), 1u << (d & 31u));
    }
}

size_t nbmask_words(int num_sites) { return ((size_t)2 * num_sites - 1 + 31) / 32; }

// The same bitmap for implicit neighbours: `row` computed neighbours per site.
__global__ void nbmask_implicit_kernel(const SearchConst c, int row, uint32_t *mask)
{
    const int64_t total = (int64_t)c.num_sites * row;
    for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < total; x += (int64_t)gridDim.x * blockDim.x) {
        const int s = (int)(x / row), e = (int)(x % row);
        const int n = lattice_neighbor(c.lat, lattice_cell(c.lat, s), e);
        const uint32_t d = (uint32_t)(n - s + c.num_sites - 1);
        atomicOr(mask + (d >> 5), 1u << (d & 31u));
    }
}

// Neighbours per site the implicit rows hold for the first S shells.
int implicit_row(const SearchConst &c, int S) { return c.lat.zoff[S - 1] + c.lat.zsize[S - 1]; }

__global__ void gather_rows_kernel(const uint8_t *occ, const int32_t *order, int count, int stride, int n,
                                   const double *f2, uint8_t *out, double *out_f2)
{
    const int p = blockIdx.y;
    if (p >= count) return;
    const uint8_t *src = occ + (size_t)order[p] * stride;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) out[(size_t)p * n + s] = src[s];
    if (blockIdx.x == 0 && threadIdx.x == 0) out_f2[p] = f2[order[p]];
}

__global__ void scatter_rows_kernel(const uint8_t *in, int count, int stride, int n, uint8_t *occ)
{
    const int p = blockIdx.y;
    if (p >= count) return;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x)
        occ[(size_t)p * stride + s] = in[(size_t)p * n + s];
}

__global__ void iota_kernel(int32_t *order, int count)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) order[i] = i;
}

// ---------------------------------------------------------------------------
// Lattice neighbour tables (pyhea/lattice/lattice.py:146-323)
// Positions in half lattice units; site id = nb * (x L^2 + y L + z) + basis.
// ---------------------------------------------------------------------------
struct LatticeSpec {
    int nb;                // basis sites per cell
    int basis[4][3];       // basis offsets, half units
    int nshell, size[3];   // shells
    int vec[3][24][3];     // offsets per shell, half units
};

__device__ __forceinline__ int basis_of(const LatticeSpec &sp, int px, int py, int pz)
{
    for (int b = 0; b < sp.nb; ++b)
        if ((sp.basis[b][0] & 1) == (px & 1) && (sp.basis[b][1] & 1) == (py & 1) && (sp.basis[b][2] & 1) == (pz & 1))
            return b;
    return -1;
}

__global__ void build_neighbors_kernel(LatticeSpec sp, int L, int32_t *out, int row, int *err)
{
    const int n = sp.nb * L * L * L;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        const int b = s % sp.nb, cell = s / sp.nb;
        const int cx = cell / (L * L), cy = (cell / L) % L, cz = cell % L;
        const int px = 2 * cx + sp.basis[b][0], py = 2 * cy + sp.basis[b][1], pz = 2 * cz + sp.basis[b][2];
        int32_t *o = out + (size_t)s * row;
        for (int k = 0; k < sp.nshell; ++k) {
            int ids[24];
            for (int v = 0; v < sp.size[k]; ++v) {
                const int qx = ((px + sp.vec[k][v][0]) % (2 * L) + 2 * L) % (2 * L);
                const int qy = ((py + sp.vec[k][v][1]) % (2 * L) + 2 * L) % (2 * L);
                const int qz = ((pz + sp.vec[k][v][2]) % (2 * L) + 2 * L) % (2 * L);
                const int nb = basis_of(sp, qx, qy, qz);
                if (nb < 0) {
                    atomicOr(err, 1);
                    ids[v] = 0;
                    continue;
                }
                ids[v] = sp.nb * ((qx >> 1) * L * L + (qy >> 1) * L + (qz >> 1)) + nb;
            }
            for (int i = 1; i < sp.size[k]; ++i) {  // ascending, as np.sort
                const int x = ids[i];
                int j = i - 1;
                while (j >= 0 && ids[j] > x) {
                    ids[j + 1] = ids[j];
                    --j;
                }
                ids[j + 1] = x;
            }
            for (int v = 0; v < sp.size[k]; ++v) o[v] = ids[v];
            o += sp.size[k];
        }
    }
}

// Sets *mismatch unless the first S shells of every site's row in `raw`
// ([N][raw_row], shells concatenated) hold the ids build_neighbors_kernel
// gives for the lattice, in any order within a shell (both sides sorted
// before the comparison).
__global__ void lattice_match_kernel(LatticeSpec sp, int L, int S, const int32_t *raw, int raw_row, int *mismatch)
{
    const int n = sp.nb * L * L * L;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        const int b = s % sp.nb, cell = s / sp.nb;
        const int cx = cell / (L * L), cy = (cell / L) % L, cz = cell % L;
        const int px = 2 * cx + sp.basis[b][0], py = 2 * cy + sp.basis[b][1], pz = 2 * cz + sp.basis[b][2];
        const int32_t *o = raw + (size_t)s * raw_row;
        bool same = true;
        for (int k = 0; k < S && same; ++k) {
            const int z = sp.size[k];
            int ids[24], got[24];
            for (int v = 0; v < z; ++v) {
                const int qx = (px + sp.vec[k][v][0] + 2 * L) % (2 * L);
                const int qy = (py + sp.vec[k][v][1] + 2 * L) % (2 * L);
                const int qz = (pz + sp.vec[k][v][2] + 2 * L) % (2 * L);
                ids[v] = sp.nb * ((qx >> 1) * L * L + (qy >> 1) * L + (qz >> 1)) + basis_of(sp, qx, qy, qz);
                got[v] = o[v];
            }
            for (int i = 1; i < z; ++i) {  // insertion sorts, both sides
                const int x = ids[i], y = got[i];
                int j = i - 1;
                while (j >= 0 && ids[j] > x) {
                    ids[j + 1] = ids[j];
                    --j;
                }
                ids[j + 1] = x;
                j = i - 1;
                while (j >= 0 && got[j] > y) {
                    got[j + 1] = got[j];
                    --j;
                }
                got[j + 1] = y;
            }
            for (int v = 0; v < z; ++v) same = same && ids[v] == got[v];
            o += z;
        }
        if (!same) atomicOr(mismatch, 1);
    }
}

int make_lattice_spec(int lattice, int shell_set, LatticeSpec &sp)
{
    std::memset(&sp, 0, sizeof(sp));
    auto add_perms = [&](int k, int a, int b, int c) {
        // all sign/axis placements of (a, b, c) with |a|,|b|,|c| given, unique
        std::vector<std::array<int, 3>> got;
        const int base[3] = {a, b, c};
        const int perm[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
        for (auto &p : perm)
            for (int sx = -1; sx <= 1; sx += 2)
                for (int sy = -1; sy <= 1; sy += 2)
                    for (int sz = -1; sz <= 1; sz += 2) {
                        std::array<int, 3> v = {sx * base[p[0]], sy * base[p[1]], sz * base[p[2]]};
                        bool dup = false;
                        for (auto &u : got) dup = dup || (u == v);
                        if (!dup) got.push_back(v);
                    }
        sp.size[k] = (int)got.size();
        for (size_t i = 0; i < got.size(); ++i)
            for (int d = 0; d < 3; ++d) sp.vec[k][i][d] = got[i][d];
    };
    sp.nshell = 3;
    if (lattice == 0) {  // FCC, lattice.py:168-194,261-323
        sp.nb = 4;
        const int bs[4][3] = {{0, 0, 0}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}};
        std::memcpy(sp.basis, bs, sizeof(bs));
        add_perms(0, 1, 1, 0);
        add_perms(1, 2, 0, 0);
        if (shell_set == 0)
            add_perms(2, 2, 2, 0);
        else
            add_perms(2, 2, 1, 1);
    } else if (lattice == 1) {  // BCC, lattice.py:146-166,196-259
        sp.nb = 2;
        const int bs[2][3] = {{0, 0, 0}, {1, 1, 1}};
        std::memcpy(sp.basis, bs, sizeof(bs));
        add_perms(0, 1, 1, 1);
        add_perms(1, 2, 0, 0);
        add_perms(2, 2, 2, 0);
    } else {
        return fail(HEA_ERR_INVALID, "lattice must be 0 (FCC) or 1 (BCC), got %d", lattice);
    }
    return HEA_OK;
}

// ---------------------------------------------------------------------------
// Validated problem with its device tables
// ---------------------------------------------------------------------------
struct DeviceTables {
    SearchConst c{};
    int T = 0, S = 0, N = 0;
    int64_t ncount = 0;
    int4 *nbor = nullptr;
    uint32_t *nbmask = nullptr;  // neighbour-offset bitmap (nbmask_kernel)
    size_t smem_gen = 0, smem_mc = 0;
    GenFn gen = nullptr;
    McFn mc = nullptr;
    int mc_block = 0;
    bool large = false;  // occupancy in HBM, one cluster per solution (hea_large.cuh)
    LGenFn lgen = nullptr;
    LRecFn lrec = nullptr;
    LFitFn lfit = nullptr;
    ~DeviceTables()
    {
        dev_free(nbor);
        dev_free(nbmask);
    }
};

int validate_problem(const hea_problem *pb, bool need_nbor = true)
{
    if (!pb) return fail(HEA_ERR_INVALID, "problem is NULL");
    if (pb->num_types < 1) return fail(HEA_ERR_INVALID, "element must name at least one species");
    if (pb->num_types < 2 || pb->num_types > kMaxTypes)
        return fail(HEA_ERR_UNSUPPORTED, "number of species must be 2..%d, got %d", kMaxTypes, pb->num_types);
    if (pb->num_shells < 1 || pb->num_shells > kMaxShells)
        return fail(HEA_ERR_UNSUPPORTED, "number of shells (len(weight)) must be 1..%d, got %d", kMaxShells,
                    pb->num_shells);
    const bool implicit = !pb->nbor && pb->implicit_lattice != 0;
    if (!pb->shell_sizes || (need_nbor && !pb->nbor && !implicit) || !pb->species || !pb->weight || !pb->target_sro)
        return fail(HEA_ERR_INVALID, "problem has a NULL array");
    int64_t n = 0;
    for (int t = 0; t < pb->num_types; ++t) {
        if (pb->species[t] < 1)
            return fail(HEA_ERR_INVALID, "species %d has %d atoms; every species needs at least one", t, pb->species[t]);
        n += pb->species[t];
    }
    if (n != pb->num_sites)
        return fail(HEA_ERR_INVALID, "num_sites %d differs from the sum of element counts %lld", pb->num_sites,
                    (long long)n);
    if (n < 2 || n > (int64_t)INT32_MAX / 2) return fail(HEA_ERR_INVALID, "number of sites %lld out of range", (long long)n);
    for (int k = 0; k < pb->num_shells; ++k) {
        if (pb->shell_sizes[k] < 1) return fail(HEA_ERR_INVALID, "shell %d is empty", k);
        if (((pb->shell_sizes[k] + 3) & ~3) > kMaxShellPad)
            return fail(HEA_ERR_UNSUPPORTED, "shell %d has %d neighbours; at most %d are supported", k,
                        pb->shell_sizes[k], kMaxShellPad);
        if (!std::isfinite(pb->weight[k]) || pb->weight[k] < 0)
            return fail(HEA_ERR_INVALID, "weight[%d] = %g must be finite and >= 0", k, pb->weight[k]);
        for (int x = 0; x < pb->num_types * pb->num_types; ++x)
            if (!std::isfinite(pb->target_sro[(size_t)k * pb->num_types * pb->num_types + x]))
                return fail(HEA_ERR_INVALID, "target_sro[%d][%d] is not finite", k, x);
    }
    if (implicit) {  // the lattice stands for the table: it must describe this structure
        if (pb->implicit_lattice < 1 || pb->implicit_lattice > 2)
            return fail(HEA_ERR_INVALID, "implicit_lattice must be 1 (FCC) or 2 (BCC), got %d", pb->implicit_lattice);
        if (pb->lattice_shell_set < 0 || pb->lattice_shell_set > 1)
            return fail(HEA_ERR_INVALID, "lattice_shell_set must be 0 or 1, got %d", pb->lattice_shell_set);
        const int64_t L = pb->lattice_cell, nb = pb->implicit_lattice == 1 ? 4 : 2;
        if (L < 2 || L > 1024 || nb * L * L * L != n)
            return fail(HEA_ERR_INVALID, "a %s cube of edge %lld does not hold %lld sites",
                        pb->implicit_lattice == 1 ? "FCC" : "BCC", (long long)L, (long long)n);
        LatticeSpec sp;
        HEA_TRY(make_lattice_spec(pb->implicit_lattice - 1, pb->lattice_shell_set, sp));
        for (int k = 0; k < pb->num_shells; ++k)
            if (pb->shell_sizes[k] != sp.size[k])
                return fail(HEA_ERR_INVALID, "shell %d of that lattice has %d neighbours, shell_sizes says %d", k,
                            sp.size[k], pb->shell_sizes[k]);
    }
    return HEA_OK;
}

// Lattice descriptor of an implicit-neighbour problem (validated), or L = 0.
void fill_lattice_const(const hea_problem *pb, SearchConst &c)
{
    std::memset(&c.lat, 0, sizeof(c.lat));
    if (pb->nbor || pb->implicit_lattice == 0) return;
    LatticeSpec sp;
    make_lattice_spec(pb->implicit_lattice - 1, pb->lattice_shell_set, sp);
    LatticeConst &lc = c.lat;
    lc.L = pb->lattice_cell;
    lc.nb = sp.nb;
    for (int k = 0, e = 0; k < 3; e += sp.size[k], ++k) {
        lc.zoff[k] = e;
        lc.zsize[k] = sp.size[k];
    }
    lc.inv_L = 1.0 / lc.L;
    lc.inv_LL = 1.0 / ((double)lc.L * lc.L);
    lc.kind = pb->implicit_lattice == 2 ? kLatBcc : pb->lattice_shell_set == 1 ? kLatFccTrue3 : kLatFccRef;
    for (int k = 0; k < kMaxShells; ++k) c.pad[k] = 0;  // no sentinel padding in computed rows
}

int validate_params(const hea_params *pr)
{
    if (!pr) return fail(HEA_ERR_INVALID, "params is NULL");
    if (pr->num_solutions < 1 || pr->num_solutions > 65535)
        return fail(HEA_ERR_INVALID, "nnet must be 1..65535, got %d", pr->num_solutions);
    if (pr->total_iter < 0 || pr->total_iter > 32766)
        return fail(HEA_ERR_INVALID, "step must be 0..32766, got %d", pr->total_iter);
    if (pr->parallel_task < 1) return fail(HEA_ERR_INVALID, "task must be >= 1, got %d", pr->parallel_task);
    if (pr->converge_depth < 0) return fail(HEA_ERR_INVALID, "depth must be >= 0, got %d", pr->converge_depth);
    return HEA_OK;
}

int smem_limit()
{
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    return v;
}

// Dynamic shared memory of mc_kernel: occupancy + sentinel, then the search's
// delta table, swap records and count buffers.
size_t mc_smem(int occ_stride, int T, int S, int nwarps)
{
    return (size_t)occ_stride + 16 + search_smem_tail(T, S, nwarps);
}

int choose_block(int tasks)
{
    int b = ((tasks + 31) / 32) * 32;
    if (b > 512) b = 512;
    return b;
}

// Kernels are shared by every plan and batch: allow them the device's largest
// dynamic shared memory (the opt-in limit less their static shared memory),
// never one plan's size.
template <class F>
cudaError_t allow_max_smem(F *func)
{
    cudaFuncAttributes a;
    cudaError_t e = cudaFuncGetAttributes(&a, func);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_limit() - (int)a.sharedSizeBytes);
}

// Search constants and padded-table geometry of a validated problem.
void fill_const(const hea_problem *pb, uint64_t seed, SearchConst &c, PadGeom &g)
{
    const int T = pb->num_types, S = pb->num_shells, N = pb->num_sites;
    std::memset(&c, 0, sizeof(c));
    g = PadGeom{};
    int raw_row = 0;
    for (int k = 0; k < S; ++k) raw_row += pb->shell_sizes[k];
    int off = 0, poff = 0;
    for (int k = 0; k < S; ++k) {
        const int z = pb->shell_sizes[k], zp = (z + 3) & ~3;
        g.size[k] = z;
        g.off[k] = off;
        g.poff[k] = poff;
        g.psize[k] = zp;
        c.off4[k] = poff / 4;
        c.chunks[k] = zp / 4;
        c.pad[k] = zp - z;
        off += z;
        poff += zp;
    }
    g.num_shells = S;
    g.raw_row = raw_row;
    g.pad_row = poff;
    g.num_sites = N;
    c.row4 = poff / 4;
    c.num_sites = N;
    c.num_types = T;
    c.num_shells = S;
    c.occ_stride = (N + 1 + 15) & ~15;  // room for the sentinel byte N in HBM rows too
    c.feistel_h = feistel_half_bits((uint32_t)N);
    c.reject_below = (uint32_t)(0u - (uint32_t)N) % (uint32_t)N;
    c.draw16 = use_draw16((uint32_t)N) ? 1u : 0u;
    c.reject16 = c.draw16 ? 65536u % (uint32_t)N : 0u;
    c.key0 = (uint32_t)seed;
    c.key1 = (uint32_t)(seed >> 32);
    c.prefix[0] = 0;
    for (int t = 0; t < T; ++t) c.prefix[t + 1] = c.prefix[t] + pb->species[t];
    for (int k = 0; k < S; ++k) {
        c.w[k] = pb->weight[k];
        for (int i = 0; i < T; ++i)
            for (int j = 0; j < T; ++j) {
                const int e = (k * T + i) * T + j;
                c.E[e] = 1.0 - pb->target_sro[(size_t)k * T * T + i * T + j];
                c.R[e] = (double)N / (((double)pb->shell_sizes[k] * (double)pb->species[i]) * (double)pb->species[j]);
            }
    }
    fill_lattice_const(pb, c);
}

// Whether a structure streams its histogram loads (SearchConst::hist_stream).
// `total_bytes` is the histogram memory of every structure resident with it
// (its own alone for a plan).  Until that total passes twice the L2 size the
// structures keep their lines cached; beyond it, those with more than
// kSharedStreamBytes of their own stream, so that the lines of the smaller
// ones stay.  Measured: a single 131 MB structure loses 3 % by streaming; on
// the mixed batch (3.7 GB) thresholds of 4, 16 and 64 MiB are within 0.4 %.
constexpr size_t kSharedStreamBytes = (size_t)64 << 20;

uint32_t stream_histograms(size_t hist_bytes, size_t total_bytes)
{
    int dev = 0, l2 = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev);
    if (total_bytes <= 2 * (size_t)l2) return 0u;
    return hist_bytes > kSharedStreamBytes ? 1u : 0u;
}

// The FCC/BCC cube whose table `pb` may pass (implicit_lattice code 1 FCC,
// 2 BCC; edge; shell set), from its site count and shell sizes alone; the
// table itself is checked on the device (lattice_match_kernel).
bool lattice_candidate(const hea_problem *pb, int &code, int &cell, int &shell_set)
{
    if (!pb->nbor || pb->implicit_lattice != 0) return false;
    const int64_t n = pb->num_sites;
    for (int lat = 0; lat < 2; ++lat) {
        const int64_t nb = lat == 0 ? 4 : 2;
        int64_t L = (int64_t)std::llround(std::cbrt((double)n / (double)nb));
        if (L < 2 || L > 1024 || nb * L * L * L != n) continue;
        for (int set = 0; set < (lat == 0 ? 2 : 1); ++set) {
            LatticeSpec sp;
            if (make_lattice_spec(lat, set, sp) != HEA_OK) continue;
            bool fits = true;
            for (int k = 0; k < pb->num_shells; ++k) fits = fits && pb->shell_sizes[k] == sp.size[k];
            if (fits) {
                code = lat + 1;
                cell = (int)L;
                shell_set = set;
                return true;
            }
        }
    }
    return false;
}

// Host twin of lattice_match_kernel, for the serving loop (which keeps a
// request's table on the host until it is placed): every site's first S
// shells of pb->nbor hold the lattice's ids, in any order within a shell.
bool table_is_lattice(const hea_problem *pb, int code, int L, int shell_set)
{
    LatticeSpec sp;
    if (make_lattice_spec(code - 1, shell_set, sp) != HEA_OK) return false;
    const int S = pb->num_shells;
    int row = 0;
    for (int k = 0; k < S; ++k) row += pb->shell_sizes[k];
    int basis_at[8];
    for (int q = 0; q < 8; ++q) basis_at[q] = -1;
    for (int b = 0; b < sp.nb; ++b)
        basis_at[((sp.basis[b][0] & 1) << 2) | ((sp.basis[b][1] & 1) << 1) | (sp.basis[b][2] & 1)] = b;
    std::vector<int32_t> ids, got;
    const int64_t n = (int64_t)sp.nb * L * L * L;
    for (int64_t s = 0; s < n; ++s) {
        const int b = (int)(s % sp.nb);
        const int64_t cell = s / sp.nb;
        const int cx = (int)(cell / ((int64_t)L * L)), cy = (int)((cell / L) % L), cz = (int)(cell % L);
        const int px = 2 * cx + sp.basis[b][0], py = 2 * cy + sp.basis[b][1], pz = 2 * cz + sp.basis[b][2];
        const int32_t *o = pb->nbor + (size_t)s * row;
        for (int k = 0; k < S; ++k) {
            const int z = sp.size[k];
            ids.resize(z);
            got.assign(o, o + z);
            for (int v = 0; v < z; ++v) {
                const int qx = (px + sp.vec[k][v][0] + 2 * L) % (2 * L);
                const int qy = (py + sp.vec[k][v][1] + 2 * L) % (2 * L);
                const int qz = (pz + sp.vec[k][v][2] + 2 * L) % (2 * L);
                ids[v] = (int32_t)(sp.nb * (((int64_t)(qx >> 1) * L + (qy >> 1)) * L + (qz >> 1)) +
                                   basis_at[((qx & 1) << 2) | ((qy & 1) << 1) | (qz & 1)]);
            }
            std::sort(ids.begin(), ids.end());
            std::sort(got.begin(), got.end());
            if (ids != got) return false;
            o += z;
        }
    }
    return true;
}

int build_tables(const hea_problem *pb, uint64_t seed, DeviceTables &dt, int32_t flags = 0)
{
    HEA_TRY(validate_problem(pb));
    const int T = pb->num_types, S = pb->num_shells, N = pb->num_sites;
    dt.T = T;
    dt.S = S;
    dt.N = N;
    dt.ncount = (int64_t)S * T * T;
    SearchConst &c = dt.c;
    PadGeom g;
    fill_const(pb, seed, c, g);
    const int raw_row = g.raw_row, poff = g.pad_row;
    const size_t raw_bytes = (size_t)N * raw_row * sizeof(int32_t);
    struct Raw {  // the uploaded table, freed on every return
        int32_t *p = nullptr;
        ~Raw() { dev_free(p); }
    } raw;

    // a table that is an FCC/BCC cube's (PyHEA's lattice tables are) runs on lattice arithmetic
    int code = 0, cell = 0, shell_set = 0;
    if (lattice_candidate(pb, code, cell, shell_set)) {
        LatticeSpec sp;
        HEA_TRY(make_lattice_spec(code - 1, shell_set, sp));
        struct Flag {
            void *p = nullptr;
            ~Flag() { dev_free(p); }
        } flag;
        int mismatch = 1;
        if (dev_alloc(&raw.p, raw_bytes) != cudaSuccess || dev_alloc(&flag.p, sizeof(int)) != cudaSuccess)
            return fail(HEA_ERR_NOMEM, "cannot allocate %zu bytes for the neighbour table", raw_bytes);
        cudaError_t e = cudaMemcpy(raw.p, pb->nbor, raw_bytes, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemset(flag.p, 0, sizeof(int));
        if (e == cudaSuccess) {
            lattice_match_kernel<<<1184, 256>>>(sp, cell, S, raw.p, raw_row, static_cast<int *>(flag.p));
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpy(&mismatch, flag.p, sizeof(int), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return fail(HEA_ERR_CUDA, "neighbour table upload failed: %s", cudaGetErrorString(e));
        if (!mismatch) {
            hea_problem q = *pb;
            q.nbor = nullptr;
            q.implicit_lattice = code;
            q.lattice_cell = cell;
            q.lattice_shell_set = shell_set;
            fill_lattice_const(&q, c);
        }
    }

    // shared memory of the two kernels
    const size_t cnt_bytes = 4 * (size_t)((dt.ncount + 3) & ~3);
    dt.smem_gen = (size_t)c.occ_stride + 16 + cnt_bytes;
    dt.smem_mc = mc_smem(c.occ_stride, T, S, 16);  // the largest block (512 threads)
    if (dt.smem_mc > (size_t)smem_limit() || (flags & HEA_FLAG_HBM_OCCUPANCY)) {
        // structures beyond shared memory: occupancy in HBM, cluster search
        dt.large = true;
        dt.mc = pick_mc_large(T, c.chunks[0], S > 1 ? c.chunks[1] : 0, S > 2 ? c.chunks[2] : 0, S, c.lat.L > 0);
        dt.lgen = kLGen[T];
        dt.lrec = kLRec[T][S];
        dt.lfit = kLFit[T][S];
        HEA_CUDA(allow_max_smem(dt.mc));
    } else {
        dt.gen = kGen[T][S];
        dt.mc = pick_mc(T, c.chunks[0], S > 1 ? c.chunks[1] : 0, S > 2 ? c.chunks[2] : 0, S, c.lat.L > 0);
        HEA_CUDA(allow_max_smem(dt.gen));
        HEA_CUDA(allow_max_smem(dt.mc));
    }

    if (c.lat.L) {  // implicit neighbours: no table, the bitmap from lattice arithmetic
        const size_t words = nbmask_words(N);
        if (dev_alloc(&dt.nbmask, words * sizeof(uint32_t)) != cudaSuccess)
            return fail(HEA_ERR_NOMEM, "cannot allocate the neighbour-offset bitmap");
        HEA_CUDA(cudaMemset(dt.nbmask, 0, words * sizeof(uint32_t)));
        nbmask_implicit_kernel<<<1184, 256>>>(c, implicit_row(c, S), dt.nbmask);
        HEA_CUDA(cudaGetLastError());
        HEA_CUDA(cudaStreamSynchronize(0));
        return HEA_OK;
    }

    // padded table on the device, checked
    const size_t pad_bytes = (size_t)N * poff * sizeof(int32_t);
    int *derr = nullptr;
    const bool uploaded = raw.p != nullptr;  // by the lattice check
    if (!uploaded) HEA_CUDA(dev_alloc(&raw.p, raw_bytes));
    if (dev_alloc(&dt.nbor, pad_bytes) != cudaSuccess || dev_alloc(&derr, sizeof(int)) != cudaSuccess) {
        dev_free(derr);
        return fail(HEA_ERR_NOMEM, "cannot allocate %zu bytes for the neighbour table", pad_bytes);
    }
    int herr = 0;
    cudaError_t e = uploaded ? cudaSuccess : cudaMemcpy(raw.p, pb->nbor, raw_bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(derr, 0, sizeof(int));
    if (e == cudaSuccess) {
        pad_and_check_kernel<<<1184, 256>>>(raw.p, reinterpret_cast<int32_t *>(dt.nbor), g, derr);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost);
    dev_free(derr);
    if (e != cudaSuccess) return fail(HEA_ERR_CUDA, "neighbour table upload failed: %s", cudaGetErrorString(e));
    if (herr & 1) return fail(HEA_ERR_INVALID, "neighbour list holds an id outside [0, %d)", N);
    if (herr & 2) return fail(HEA_ERR_UNSUPPORTED, "neighbour list names a site as its own neighbour");
    if (herr & 4)
        return fail(HEA_ERR_UNSUPPORTED,
                    "neighbour list is not symmetric within a shell (site a lists b a different number of times "
                    "than b lists a)");
    const size_t words = nbmask_words(N);
    if (dev_alloc(&dt.nbmask, words * sizeof(uint32_t)) != cudaSuccess)
        return fail(HEA_ERR_NOMEM, "cannot allocate the neighbour-offset bitmap");
    HEA_CUDA(cudaMemset(dt.nbmask, 0, words * sizeof(uint32_t)));
    nbmask_kernel<<<1184, 256>>>(reinterpret_cast<const int32_t *>(dt.nbor), N, poff, dt.nbmask);
    HEA_CUDA(cudaGetLastError());
    HEA_CUDA(cudaStreamSynchronize(0));  // callers launch on their own non-blocking streams
    return HEA_OK;
}

struct DeviceBuf {
    void *p = nullptr;
    ~DeviceBuf() { dev_free(p); }
};

}  // namespace

// ---------------------------------------------------------------------------
// Plan
// ---------------------------------------------------------------------------
struct hea_plan {
    DeviceTables dt;
    hea_params prm{};
    int P = 0;
    cudaStream_t stream = nullptr, side = nullptr;  // side: the next iteration's new population
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::vector<cudaEvent_t> joins;  // fork/join events between the two streams
    uint8_t *occ = nullptr, *out_occ = nullptr;
    int32_t *cnt = nullptr, *order = nullptr, *scratch = nullptr;
    double *f2 = nullptr, *out_f2 = nullptr;
    uint4 *hist = nullptr;  // [slots][N] site histograms
    unsigned long long *stats = nullptr;
    std::vector<cudaEvent_t> mc_events;  // start/stop pairs, HEA_FLAG_TIME_KERNELS
    int mc_timed = 0;
    int mc_block = 0;  // threads per CTA of the local search (choose_block, or the autotuner's pick)
    // HEA_FLAG_LOG_ITERS: each iteration's best f2 written by the device into mapped pinned memory
    // and printed by a host callback on the stream (no host synchronisation per iteration)
    struct LogEntry {
        int it;
        const double *best;
    };
    double *log_host = nullptr, *log_dev = nullptr;
    std::vector<LogEntry> log_entries;
    ~hea_plan()
    {
        if (stream) cudaStreamSynchronize(stream);  // buffers return to the pool only when idle
        if (side) cudaStreamSynchronize(side);
        if (log_host) cudaFreeHost(log_host);
        for (cudaEvent_t e : mc_events) cudaEventDestroy(e);
        for (cudaEvent_t e : joins) cudaEventDestroy(e);
        if (side) cudaStreamDestroy(side);
        for (void *p : {(void *)occ, (void *)out_occ, (void *)cnt, (void *)order, (void *)scratch, (void *)f2,
                        (void *)out_f2, (void *)stats, (void *)hist})
            dev_free(p);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

int launch_generate(hea_plan *pl, const int32_t *order, int count, uint32_t generation, int generate,
                    cudaStream_t st = nullptr)
{
    if (!st) st = pl->stream;
    GenArgs a{};
    a.nbor = pl->dt.nbor;
    a.occ = pl->occ;
    a.cnt = pl->cnt;
    a.f2 = pl->f2;
    a.order = order;
    a.generation = generation;
    a.generate = generate;
    a.hist = pl->hist;
    if (pl->dt.large) {
        const SearchConst &c = pl->dt.c;
        int chunks = (c.num_sites + 255) / 256;
        const int cap = std::max(1, 2368 / count);
        if (chunks > cap) chunks = cap;
        zero_counts_kernel<<<dim3(1, count), 128, 0, st>>>(order, count, pl->cnt, (int)pl->dt.ncount);
        if (generate) pl->dt.lgen<<<dim3(chunks, count), 256, 0, st>>>(c, pl->occ, order, generation);
        pl->dt.lrec<<<dim3(chunks, count), 256, 0, st>>>(c, pl->dt.nbor, pl->occ, order, pl->cnt, pl->hist);
        pl->dt.lfit<<<(count + 127) / 128, 128, 0, st>>>(c, order, count, pl->cnt, pl->f2);
        HEA_CUDA(cudaGetLastError());
        return HEA_OK;
    }
    pl->dt.gen<<<count, 512, pl->dt.smem_gen, st>>>(pl->dt.c, a);
    HEA_CUDA(cudaGetLastError());
    return HEA_OK;
}

int launch_mc(hea_plan *pl, const int32_t *order, int count, uint32_t mc_call, McArgs extra, cudaStream_t st = nullptr)
{
    if (!st) st = pl->stream;
    McArgs a = extra;
    a.nbor = pl->dt.nbor;
    a.occ = pl->occ;
    a.cnt = pl->cnt;
    a.f2 = pl->f2;
    a.order = order;
    a.hist = pl->hist;
    a.nbmask = pl->dt.nbmask;
    a.mc_call = mc_call;
    a.tasks = pl->prm.parallel_task;
    a.depth = pl->prm.converge_depth;
    a.max_rounds = pl->prm.max_rounds > 0 ? pl->prm.max_rounds : (int64_t)1 << 31;
    a.stats = pl->stats;
    const bool timed = (pl->prm.flags & HEA_FLAG_TIME_KERNELS) && 2 * pl->mc_timed + 1 < (int)pl->mc_events.size();
    if (timed) HEA_CUDA(cudaEventRecord(pl->mc_events[2 * pl->mc_timed], st));
    if (pl->dt.large) {
        // one cluster of up to 8 CTAs per solution, each with a share of the tasks
        int csize = (a.tasks + 511) / 512;
        csize = csize < 1 ? 1 : (csize > 8 ? 8 : csize);
        const int block = choose_block((a.tasks + csize - 1) / csize);
        const int nw = block / 32;
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3(count * csize);
        cfg.blockDim = dim3(block);
        cfg.dynamicSmemBytes = search_smem_tail(pl->dt.T, pl->dt.S, nw) + 2 * sizeof(SwapRecord);
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = csize;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        HEA_CUDA(cudaLaunchKernelEx(&cfg, pl->dt.mc, pl->dt.c, a));
    } else {
        const int block = pl->mc_block;
        pl->dt.mc<<<count, block, mc_smem(pl->dt.c.occ_stride, pl->dt.T, pl->dt.S, block / 32), st>>>(pl->dt.c, a);
    }
    HEA_CUDA(cudaGetLastError());
    if (timed) {
        HEA_CUDA(cudaEventRecord(pl->mc_events[2 * pl->mc_timed + 1], st));
        ++pl->mc_timed;
    }
    return HEA_OK;
}

int launch_sort(hea_plan *pl, int32_t *order, int count)
{
    sort_slots_kernel<<<1, 1024, 0, pl->stream>>>(order, pl->f2, count, pl->scratch);
    HEA_CUDA(cudaGetLastError());
    return HEA_OK;
}

int plan_alloc(hea_plan *pl, int slots)
{
    const SearchConst &c = pl->dt.c;
    HEA_CUDA(cudaStreamCreateWithFlags(&pl->stream, cudaStreamNonBlocking));
    HEA_CUDA(cudaStreamCreateWithFlags(&pl->side, cudaStreamNonBlocking));
    for (int i = 0; i < 2; ++i) {
        cudaEvent_t e;
        HEA_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        pl->joins.push_back(e);
    }
    HEA_CUDA(cudaEventCreate(&pl->ev0));
    HEA_CUDA(cudaEventCreate(&pl->ev1));
    const size_t occ_bytes = (size_t)slots * c.occ_stride;
    if (dev_alloc(&pl->occ, occ_bytes) != cudaSuccess ||
        dev_alloc(&pl->cnt, (size_t)slots * pl->dt.ncount * sizeof(int32_t)) != cudaSuccess ||
        dev_alloc(&pl->order, (size_t)slots * sizeof(int32_t)) != cudaSuccess ||
        dev_alloc(&pl->scratch, (size_t)slots * sizeof(int32_t)) != cudaSuccess ||
        dev_alloc(&pl->f2, (size_t)slots * sizeof(double)) != cudaSuccess ||
        dev_alloc(&pl->out_occ, (size_t)slots * c.num_sites) != cudaSuccess ||
        dev_alloc(&pl->out_f2, (size_t)slots * sizeof(double)) != cudaSuccess ||
        dev_alloc(&pl->stats, 4 * sizeof(unsigned long long)) != cudaSuccess)
        return fail(HEA_ERR_NOMEM, "cannot allocate the population buffers (%zu bytes of occupancy)", occ_bytes);
    if (dev_alloc(&pl->hist, (size_t)slots * c.num_sites * sizeof(uint4)) != cudaSuccess)
        return fail(HEA_ERR_NOMEM, "cannot allocate the site histograms (%zu bytes)",
                    (size_t)slots * c.num_sites * sizeof(uint4));
    HEA_CUDA(cudaMemsetAsync(pl->occ, 0, occ_bytes, pl->stream));
    iota_kernel<<<(slots + 255) / 256, 256, 0, pl->stream>>>(pl->order, slots);
    HEA_CUDA(cudaGetLastError());
    return HEA_OK;
}

void log_iteration(int it, double best)
{
    std::time_t now = std::time(nullptr);
    char ts[32];
    std::strftime(ts, sizeof(ts), "%Y-%m-%d %H:%M:%S", std::localtime(&now));
    std::printf("%s - PyHEA - INFO - Iter %d with best fitness:      %g\n", ts, it, best);
    std::fflush(stdout);
}

// The best f2 of a sorted population (slot order[0]) into *out (mapped pinned memory).
__global__ void best_f2_kernel(const int32_t *order, const double *f2, double *out) { *out = f2[order[0]]; }

// Stream host callback: prints the log line of one iteration once the device
// has written its best f2 (no CUDA calls here).
void CUDART_CB log_callback(void *arg)
{
    const hea_plan::LogEntry *e = static_cast<const hea_plan::LogEntry *>(arg);
    log_iteration(e->it, std::sqrt(*e->best));
}

// Mapped pinned memory for one best f2 per iteration (HEA_FLAG_LOG_ITERS).
int plan_log_buffers(hea_plan *pl)
{
    const int I = pl->prm.total_iter;
    if (!(pl->prm.flags & HEA_FLAG_LOG_ITERS) || I < 1 || (int)pl->log_entries.size() >= I) return HEA_OK;
    if (pl->log_host) {
        HEA_CUDA(cudaStreamSynchronize(pl->stream));
        cudaFreeHost(pl->log_host);
        pl->log_host = nullptr;
    }
    HEA_CUDA(cudaHostAlloc((void **)&pl->log_host, sizeof(double) * I, cudaHostAllocMapped));
    HEA_CUDA(cudaHostGetDevicePointer((void **)&pl->log_dev, pl->log_host, 0));
    pl->log_entries.resize(I);
    for (int it = 0; it < I; ++it) pl->log_entries[it] = hea_plan::LogEntry{it, pl->log_host + it};
    return HEA_OK;
}

int read_population(hea_plan *pl, int count, uint8_t *out_occ, double *out_fitness)
{
    const SearchConst &c = pl->dt.c;
    dim3 grid((c.num_sites + 255) / 256 < 64 ? (c.num_sites + 255) / 256 : 64, count);
    gather_rows_kernel<<<grid, 256, 0, pl->stream>>>(pl->occ, pl->order, count, c.occ_stride, c.num_sites, pl->f2,
                                                     pl->out_occ, pl->out_f2);
    HEA_CUDA(cudaGetLastError());
    if (out_occ)
        HEA_CUDA(cudaMemcpyAsync(out_occ, pl->out_occ, (size_t)count * c.num_sites, cudaMemcpyDeviceToHost, pl->stream));
    std::vector<double> f(count);
    HEA_CUDA(cudaMemcpyAsync(f.data(), pl->out_f2, count * sizeof(double), cudaMemcpyDeviceToHost, pl->stream));
    HEA_CUDA(cudaStreamSynchronize(pl->stream));
    if (out_fitness)
        for (int p = 0; p < count; ++p) out_fitness[p] = std::sqrt(f[p]);
    return HEA_OK;
}

// The global loop of accelerate.cpp:737-761: generation 0, then per iteration a
// new population searched (call 2*it), merged (stable, current first), and the
// survivors searched (call 2*it+1) and sorted.
int plan_search(hea_plan *pl, hea_stats *stats)
{
    const int P = pl->P;
    pl->mc_timed = 0;
    if ((pl->prm.flags & HEA_FLAG_TIME_KERNELS) && pl->mc_events.size() < (size_t)(4 * pl->prm.total_iter)) {
        while (pl->mc_events.size() < (size_t)(4 * pl->prm.total_iter)) {
            cudaEvent_t e;
            HEA_CUDA(cudaEventCreate(&e));
            pl->mc_events.push_back(e);
        }
    }
    HEA_TRY(plan_log_buffers(pl));
    HEA_CUDA(cudaMemsetAsync(pl->stats, 0, 4 * sizeof(unsigned long long), pl->stream));
    iota_kernel<<<(2 * P + 255) / 256, 256, 0, pl->stream>>>(pl->order, 2 * P);
    HEA_CUDA(cudaGetLastError());
    HEA_CUDA(cudaEventRecord(pl->ev0, pl->stream));
    HEA_TRY(launch_generate(pl, pl->order, P, 0, 1));
    const int I = pl->prm.total_iter;
    if (I > 0) {
        HEA_TRY(launch_generate(pl, pl->order + P, P, 1, 1));
        HEA_TRY(launch_mc(pl, pl->order + P, P, 0, McArgs{}));
        HEA_TRY(launch_sort(pl, pl->order, 2 * P));
    }
    for (int it = 0; it < I; ++it) {
        // after the merge of iteration it, the new population of iteration it+1
        // (free slots order[P, 2P)) is generated and searched on the side stream
        // while the survivors (order[0, P)) are searched on the main stream
        if (it + 1 < I) {
            HEA_CUDA(cudaEventRecord(pl->joins[0], pl->stream));
            HEA_CUDA(cudaStreamWaitEvent(pl->side, pl->joins[0], 0));
            HEA_TRY(launch_generate(pl, pl->order + P, P, (uint32_t)(it + 2), 1, pl->side));
            HEA_TRY(launch_mc(pl, pl->order + P, P, (uint32_t)(2 * (it + 1)), McArgs{}, pl->side));
            HEA_CUDA(cudaEventRecord(pl->joins[1], pl->side));
        }
        HEA_TRY(launch_mc(pl, pl->order, P, (uint32_t)(2 * it + 1), McArgs{}));
        HEA_TRY(launch_sort(pl, pl->order, P));
        if (pl->prm.flags & HEA_FLAG_LOG_ITERS) {  // the reference's per-iteration line (accelerate.cu:1208-1212)
            best_f2_kernel<<<1, 1, 0, pl->stream>>>(pl->order, pl->f2, pl->log_dev + it);
            HEA_CUDA(cudaGetLastError());
            HEA_CUDA(cudaLaunchHostFunc(pl->stream, log_callback, &pl->log_entries[it]));
        }
        if (it + 1 < I) {
            HEA_CUDA(cudaStreamWaitEvent(pl->stream, pl->joins[1], 0));
            HEA_TRY(launch_sort(pl, pl->order, 2 * P));  // merge of iteration it+1
        }
    }
    HEA_CUDA(cudaEventRecord(pl->ev1, pl->stream));
    HEA_CUDA(cudaStreamSynchronize(pl->stream));
    if (stats) {
        unsigned long long s[4];
        HEA_CUDA(cudaMemcpy(s, pl->stats, sizeof(s), cudaMemcpyDeviceToHost));
        float ms = 0;
        HEA_CUDA(cudaEventElapsedTime(&ms, pl->ev0, pl->ev1));
        stats->rounds = (int64_t)s[0];
        stats->evals = (int64_t)s[1];
        stats->accepts = (int64_t)s[2];
        stats->gpu_ms = ms;
        // local-search busy time: union of the launch intervals (launches on
        // the two streams overlap), from event times relative to ev0
        std::vector<std::pair<float, float>> iv;
        for (int i = 0; i < pl->mc_timed; ++i) {
            float a = 0, b = 0;
            HEA_CUDA(cudaEventElapsedTime(&a, pl->ev0, pl->mc_events[2 * i]));
            HEA_CUDA(cudaEventElapsedTime(&b, pl->ev0, pl->mc_events[2 * i + 1]));
            iv.emplace_back(a, b);
        }
        std::sort(iv.begin(), iv.end());
        double busy = 0, lo = 0, hi = -1;
        for (auto &x : iv) {
            if (x.first > hi) {
                if (hi > lo) busy += hi - lo;
                lo = x.first;
                hi = x.second;
            } else if (x.second > hi) {
                hi = x.second;
            }
        }
        if (hi > lo) busy += hi - lo;
        stats->mc_ms = busy;
        stats->mc_launches = pl->mc_timed;
    }
    return HEA_OK;
}

// Autotuner of the local search's CTA size.  Every CTA size gives the same
// result (the round's winner is the lexicographic (f2, task) minimum however
// the tasks are split over warps and passes), so the choice is a pure speed
// question: each candidate (the default one task per thread, and 256 and 128
// threads when smaller) searches a fresh generation-0 population for
// kTuneRounds rounds, once to warm up and kTunePasses times timed; a
// candidate's rate is its best pass (evaluations per millisecond).  A smaller
// CTA replaces the default only when its rate is above the default's by more
// than kTuneMargin, so timing noise cannot trade the default for a near tie.
// Picks are cached per device and shape for the life of the process.
struct TuneKey {
    int dev, N, T, S, row4, Q, P;
    bool operator<(const TuneKey &o) const
    {
        return std::tie(dev, N, T, S, row4, Q, P) < std::tie(o.dev, o.N, o.T, o.S, o.row4, o.Q, o.P);
    }
};
std::mutex g_tune_mu;
std::map<TuneKey, int> g_tune;
constexpr int kTuneRounds = 200;
constexpr int kTunePasses = 3;
constexpr double kTuneMargin = 1.05;

// With measure = false only a cached pick is applied (plans created without
// HEA_FLAG_AUTOTUNE still use the pick of an earlier tuned plan of their shape).
int plan_autotune(hea_plan *pl, bool measure)
{
    if (pl->dt.large) return HEA_OK;  // cluster size follows the task count
    const SearchConst &c = pl->dt.c;
    int dev = 0;
    HEA_CUDA(cudaGetDevice(&dev));
    const TuneKey key{dev, c.num_sites, pl->dt.T, pl->dt.S, c.row4, pl->prm.parallel_task, pl->P};
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune.find(key);
        if (it != g_tune.end()) {
            pl->mc_block = it->second;
            return HEA_OK;
        }
    }
    if (!measure) return HEA_OK;
    std::vector<int> cand = {choose_block(pl->prm.parallel_task)};
    for (int b : {256, 128})
        if (b < cand[0]) cand.push_back(b);
    int best = cand[0];
    if (cand.size() > 1) {
        const hea_params saved = pl->prm;
        const int64_t cap = saved.max_rounds > 0 ? std::min<int64_t>(saved.max_rounds, kTuneRounds) : kTuneRounds;
        pl->prm.max_rounds = cap;
        pl->prm.flags &= ~HEA_FLAG_TIME_KERNELS;
        std::vector<double> rate_of(cand.size(), 0.0);
        int rc = HEA_OK;
        for (int pass = 0; pass <= kTunePasses && rc == HEA_OK; ++pass) {  // pass 0 warms up
            for (size_t ci = 0; ci < cand.size(); ++ci) {
                const int b = cand[ci];
                pl->mc_block = b;
                cudaMemsetAsync(pl->stats, 0, 4 * sizeof(unsigned long long), pl->stream);
                iota_kernel<<<(2 * pl->P + 255) / 256, 256, 0, pl->stream>>>(pl->order, 2 * pl->P);
                if ((rc = launch_generate(pl, pl->order, pl->P, 0, 1)) != HEA_OK) break;
                cudaEventRecord(pl->ev0, pl->stream);
                if ((rc = launch_mc(pl, pl->order, pl->P, 0, McArgs{})) != HEA_OK) break;
                cudaEventRecord(pl->ev1, pl->stream);
                unsigned long long st[4];
                cudaError_t e = cudaMemcpyAsync(st, pl->stats, sizeof(st), cudaMemcpyDeviceToHost, pl->stream);
                if (e == cudaSuccess) e = cudaStreamSynchronize(pl->stream);
                float ms = 0;
                if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, pl->ev0, pl->ev1);
                if (e != cudaSuccess) {
                    rc = fail(HEA_ERR_CUDA, "autotuning failed: %s", cudaGetErrorString(e));
                    break;
                }
                const double rate = ms > 0 ? st[1] / (double)ms : 0.0;
                if (pass > 0) rate_of[ci] = std::max(rate_of[ci], rate);
            }
        }
        pl->prm = saved;
        if (rc != HEA_OK) return rc;
        double best_rate = rate_of[0] * kTuneMargin;  // cand[0] is the default
        for (size_t ci = 1; ci < cand.size(); ++ci)
            if (rate_of[ci] > best_rate) {
                best_rate = rate_of[ci];
                best = cand[ci];
            }
    }
    pl->mc_block = best;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[key] = best;
    return HEA_OK;
}

int plan_create(const hea_problem *pb, const hea_params *prm, int slots, hea_plan **out)
{
    *out = nullptr;
    hea_plan *pl = new (std::nothrow) hea_plan();
    if (!pl) return fail(HEA_ERR_NOMEM, "out of host memory");
    int rc = build_tables(pb, prm->seed, pl->dt, prm->flags);
    if (rc == HEA_OK) {
        pl->prm = *prm;
        pl->P = prm->num_solutions;
        pl->mc_block = choose_block(prm->parallel_task);
        rc = plan_alloc(pl, slots);
        const size_t hist_bytes = (size_t)slots * pl->dt.N * sizeof(uint4);
        pl->dt.c.hist_stream = stream_histograms(hist_bytes, hist_bytes);
    }
    if (rc == HEA_OK) rc = plan_autotune(pl, (prm->flags & HEA_FLAG_AUTOTUNE) != 0);
    if (rc != HEA_OK) {
        delete pl;
        return rc;
    }
    *out = pl;
    return HEA_OK;
}

hea_params component_params(int count, int tasks, int depth, int64_t max_rounds, uint64_t seed)
{
    hea_params p{};
    p.num_solutions = count;
    p.total_iter = 0;
    p.parallel_task = tasks;
    p.converge_depth = depth;
    p.seed = seed;
    p.max_rounds = max_rounds;
    return p;
}

}  // namespace

// ---------------------------------------------------------------------------
// Public entry points
// ---------------------------------------------------------------------------
extern "C" {

void hea_release_cached_memory(void)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return;
    DevicePool &P = pool();
    std::lock_guard<std::mutex> lk(P.mu);
    pool_release_device(P, dev);
}

int hea_cuda_available(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n > 0;
}

const char *hea_last_error(void) { return g_error.c_str(); }

}  // extern "C"

namespace {
// Reads the buffer `reps` times with 16-byte loads through L2 (four in flight
// per thread); the xor of everything read goes to *sink only if it matches a
// value it never takes in practice, so the loads are not removed.
__global__ void __launch_bounds__(256) l2_read_probe_kernel(const uint4 *buf, int64_t n16, int reps, uint32_t *sink)
{
    uint32_t acc = 0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int r = 0; r < reps; ++r)
        for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n16; i += 4 * stride) {
            uint4 v[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) v[u] = i + u * stride < n16 ? __ldcg(buf + i + u * stride) : make_uint4(0, 0, 0, 0);
#pragma unroll
            for (int u = 0; u < 4; ++u) acc ^= v[u].x ^ v[u].y ^ v[u].z ^ v[u].w;
        }
    if (acc == 0x9E3779B9u) atomicAdd(sink, 1u);
}

// Random 16-byte loads through L2 from a buffer far larger than L2, eight in
// flight per thread: the access pattern of the site-histogram loads of
// structures whose histograms do not fit in L2.  Indices come from the murmur3
// finaliser of a per-thread counter, mapped to [0, n16) by a multiply-high.
template <bool kStream>
__global__ void __launch_bounds__(256) dram_random_probe_kernel(const uint4 *buf, uint64_t n16, int per_thread,
                                                                uint32_t seed, uint32_t *sink)
{
    uint32_t acc = 0;
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    for (int i = 0; i < per_thread; i += 8) {
        uint4 v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const uint32_t h = fmix32(seed ^ (t * 0x9E3779B9u) ^ (uint32_t)(i + u) * 0x85EBCA6Bu);
            const uint64_t idx = ((uint64_t)h * n16) >> 32;
            v[u] = kStream ? __ldcs(buf + idx) : __ldcg(buf + idx);
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) acc ^= v[u].x ^ v[u].w;
    }
    if (acc == 0x9E3779B9u) atomicAdd(sink, 1u);
}
}  // namespace

extern "C" {

int hea_dram_random_probe(int64_t bytes, int32_t per_thread, double *out_loads_per_s)
{
    if (bytes < ((int64_t)1 << 28) || per_thread < 8 || per_thread % 8 || !out_loads_per_s)
        return fail(HEA_ERR_INVALID, "bytes >= 256 MiB, per_thread a positive multiple of 8, out_loads_per_s");
    int dev = 0, sms = 0;
    HEA_CUDA(cudaGetDevice(&dev));
    HEA_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const uint64_t n16 = (uint64_t)bytes / 16;
    if (n16 > 0xFFFFFFFFull) return fail(HEA_ERR_INVALID, "at most 64 GiB");
    struct Owned {  // the probe's buffer goes back to the driver, not to the block cache
        void *p = nullptr;
        ~Owned() { if (p) cudaFree(p); }
    } buf, sink;
    if (cudaMalloc(&buf.p, (size_t)n16 * 16) != cudaSuccess || cudaMalloc(&sink.p, sizeof(uint32_t)) != cudaSuccess)
        return fail(HEA_ERR_NOMEM, "cannot allocate %lld bytes for the probe", (long long)bytes);
    HEA_CUDA(cudaMemset(buf.p, 1, (size_t)n16 * 16));
    cudaEvent_t e0, e1;
    HEA_CUDA(cudaEventCreate(&e0));
    HEA_CUDA(cudaEventCreate(&e1));
    // L2-cached and evict-first loads, 8 and 32 CTAs per SM (more loads in flight); the best rate
    double best = 0.0;
    cudaError_t e = cudaSuccess;
    for (int stream = 0; stream < 2 && e == cudaSuccess; ++stream)
        for (int per_sm : {8, 32}) {
            const int grid = sms * per_sm;
            const auto kern = stream ? dram_random_probe_kernel<true> : dram_random_probe_kernel<false>;
            kern<<<grid, 256>>>((const uint4 *)buf.p, n16, 8, 1u, (uint32_t *)sink.p);
            cudaEventRecord(e0);
            kern<<<grid, 256>>>((const uint4 *)buf.p, n16, per_thread, 7u, (uint32_t *)sink.p);
            cudaEventRecord(e1);
            e = cudaEventSynchronize(e1);
            float ms = 0.0f;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
            if (e != cudaSuccess) break;
            best = std::max(best, (double)grid * 256.0 * per_thread / (ms * 1e-3));
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e != cudaSuccess) return fail(HEA_ERR_CUDA, "DRAM probe failed: %s", cudaGetErrorString(e));
    *out_loads_per_s = best;
    return HEA_OK;
}

int hea_l2_read_probe(int64_t bytes, int32_t reps, double *out_gbs)
{
    if (bytes < (1 << 20) || reps < 1 || !out_gbs) return fail(HEA_ERR_INVALID, "bytes >= 1 MiB, reps >= 1, out_gbs");
    int dev = 0, sms = 0, l2 = 0;
    HEA_CUDA(cudaGetDevice(&dev));
    HEA_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    HEA_CUDA(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev));
    if (bytes > l2) return fail(HEA_ERR_INVALID, "%lld bytes do not fit in the %d-byte L2", (long long)bytes, l2);
    const int64_t n16 = bytes / 16;
    DeviceBuf buf, sink;
    HEA_CUDA(dev_alloc(&buf.p, (size_t)n16 * 16));
    HEA_CUDA(dev_alloc(&sink.p, sizeof(uint32_t)));
    HEA_CUDA(cudaMemset(buf.p, 1, (size_t)n16 * 16));
    cudaEvent_t e0, e1;
    HEA_CUDA(cudaEventCreate(&e0));
    HEA_CUDA(cudaEventCreate(&e1));
    const int grid = sms * 8;
    l2_read_probe_kernel<<<grid, 256>>>((const uint4 *)buf.p, n16, 1, (uint32_t *)sink.p);  // brings it into L2
    cudaEventRecord(e0);
    l2_read_probe_kernel<<<grid, 256>>>((const uint4 *)buf.p, n16, reps, (uint32_t *)sink.p);
    cudaEventRecord(e1);
    cudaError_t e = cudaEventSynchronize(e1);
    float ms = 0.0f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e != cudaSuccess) return fail(HEA_ERR_CUDA, "L2 probe failed: %s", cudaGetErrorString(e));
    *out_gbs = (double)n16 * 16.0 * reps / (ms * 1e-3) / 1e9;
    return HEA_OK;
}

int hea_plan_create(const hea_problem *problem, const hea_params *params, hea_plan **out)
{
    if (!out) return fail(HEA_ERR_INVALID, "out is NULL");
    HEA_TRY(validate_params(params));
    return plan_create(problem, params, 2 * params->num_solutions, out);
}

int hea_plan_run(hea_plan *plan, uint64_t seed, hea_stats *stats)
{
    if (!plan) return fail(HEA_ERR_INVALID, "plan is NULL");
    plan->dt.c.key0 = (uint32_t)seed;
    plan->dt.c.key1 = (uint32_t)(seed >> 32);
    plan->prm.seed = seed;
    return plan_search(plan, stats);
}

int hea_plan_read(hea_plan *plan, uint8_t *out_occ, double *out_fitness)
{
    if (!plan) return fail(HEA_ERR_INVALID, "plan is NULL");
    return read_population(plan, plan->P, out_occ, out_fitness);
}

void hea_plan_destroy(hea_plan *plan) { delete plan; }

int32_t hea_plan_local_search_block(const hea_plan *plan) { return plan ? plan->mc_block : 0; }

int32_t hea_plan_lattice(const hea_plan *plan)
{
    if (!plan || plan->dt.c.lat.L == 0) return 0;
    return plan->dt.c.lat.kind == kLatBcc ? 2 : 1;
}

int hea_run_local_parallel_hcs(const hea_problem *problem, const hea_params *params, uint8_t *out_occ,
                               double *out_fitness, hea_stats *stats)
{
    hea_plan *pl = nullptr;
    HEA_TRY(hea_plan_create(problem, params, &pl));
    int rc = plan_search(pl, stats);
    if (rc == HEA_OK) rc = read_population(pl, pl->P, out_occ, out_fitness);
    delete pl;
    return rc;
}

int hea_generate(const hea_problem *problem, uint64_t seed, uint32_t generation, int32_t count, uint8_t *out_occ,
                 int32_t *out_counts, double *out_f2)
{
    if (count < 1 || count > 65535) return fail(HEA_ERR_INVALID, "count must be 1..65535");
    hea_params p = component_params(count, 1, 0, 0, seed);
    hea_plan *pl = nullptr;
    HEA_TRY(plan_create(problem, &p, count, &pl));
    int rc = launch_generate(pl, pl->order, count, generation, 1);
    if (rc == HEA_OK && out_counts) {
        cudaError_t e = cudaMemcpyAsync(out_counts, pl->cnt, (size_t)count * pl->dt.ncount * sizeof(int32_t),
                                        cudaMemcpyDeviceToHost, pl->stream);
        if (e != cudaSuccess) rc = fail(HEA_ERR_CUDA, "copy of counts failed: %s", cudaGetErrorString(e));
    }
    if (rc == HEA_OK) rc = read_population(pl, count, out_occ, nullptr);
    if (rc == HEA_OK && out_f2) {
        cudaError_t e = cudaMemcpy(out_f2, pl->f2, count * sizeof(double), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) rc = fail(HEA_ERR_CUDA, "copy of f2 failed: %s", cudaGetErrorString(e));
    }
    delete pl;
    return rc;
}

namespace {
int load_occupancy(hea_plan *pl, int count, const uint8_t *occ)
{
    const SearchConst &c = pl->dt.c;
    const int T = pl->dt.T;
    for (size_t x = 0; x < (size_t)count * c.num_sites; ++x)
        if (occ[x] >= T) return fail(HEA_ERR_INVALID, "occupancy holds species %d >= %d", occ[x], T);
    for (int p = 0; p < count; ++p) {  // composition must match element
        std::vector<int64_t> h(T, 0);
        for (int s = 0; s < c.num_sites; ++s) ++h[occ[(size_t)p * c.num_sites + s]];
        for (int t = 0; t < T; ++t)
            if (h[t] != c.prefix[t + 1] - c.prefix[t])
                return fail(HEA_ERR_INVALID, "occupancy %d has %lld atoms of species %d, element says %d", p,
                            (long long)h[t], t, c.prefix[t + 1] - c.prefix[t]);
    }
    HEA_CUDA(cudaMemcpyAsync(pl->out_occ, occ, (size_t)count * c.num_sites, cudaMemcpyHostToDevice, pl->stream));
    dim3 grid((c.num_sites + 255) / 256 < 64 ? (c.num_sites + 255) / 256 : 64, count);
    scatter_rows_kernel<<<grid, 256, 0, pl->stream>>>(pl->out_occ, count, c.occ_stride, c.num_sites, pl->occ);
    HEA_CUDA(cudaGetLastError());
    return launch_generate(pl, pl->order, count, 0, 0);
}
}  // namespace

int hea_recount(const hea_problem *problem, int32_t count, const uint8_t *occ, int32_t *out_counts, double *out_f2)
{
    if (count < 1 || count > 65535) return fail(HEA_ERR_INVALID, "count must be 1..65535");
    if (!occ) return fail(HEA_ERR_INVALID, "occ is NULL");
    hea_params p = component_params(count, 1, 0, 0, 0);
    hea_plan *pl = nullptr;
    HEA_TRY(plan_create(problem, &p, count, &pl));
    int rc = load_occupancy(pl, count, occ);
    if (rc == HEA_OK && out_counts) {
        cudaError_t e = cudaMemcpyAsync(out_counts, pl->cnt, (size_t)count * pl->dt.ncount * sizeof(int32_t),
                                        cudaMemcpyDeviceToHost, pl->stream);
        if (e != cudaSuccess) rc = fail(HEA_ERR_CUDA, "copy of counts failed: %s", cudaGetErrorString(e));
    }
    if (rc == HEA_OK) rc = read_population(pl, count, nullptr, nullptr);
    if (rc == HEA_OK && out_f2) {
        cudaError_t e = cudaMemcpy(out_f2, pl->f2, count * sizeof(double), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) rc = fail(HEA_ERR_CUDA, "copy of f2 failed: %s", cudaGetErrorString(e));
    }
    delete pl;
    return rc;
}

int hea_local_search(const hea_problem *problem, uint64_t seed, uint32_t mc_call, int32_t count, int32_t tasks,
                     int32_t depth, int64_t max_rounds, uint8_t *occ, int32_t *out_counts, double *out_f2,
                     int64_t *out_rounds, hea_accept_record *trace, int32_t *trace_counts, int64_t trace_cap,
                     int64_t *trace_len)
{
    if (count < 1 || count > 65535) return fail(HEA_ERR_INVALID, "count must be 1..65535");
    if (tasks < 1) return fail(HEA_ERR_INVALID, "tasks must be >= 1");
    if (depth < 0) return fail(HEA_ERR_INVALID, "depth must be >= 0");
    if (mc_call > 65534) return fail(HEA_ERR_INVALID, "mc_call must be <= 65534");
    if (!occ) return fail(HEA_ERR_INVALID, "occ is NULL");
    if (trace_cap < 0 || (trace_cap > 0 && (!trace || !trace_len)))
        return fail(HEA_ERR_INVALID, "trace needs trace, trace_len and trace_cap >= 0");
    hea_params p = component_params(count, tasks, depth, max_rounds, seed);
    hea_plan *pl = nullptr;
    HEA_TRY(plan_create(problem, &p, count, &pl));
    int rc = load_occupancy(pl, count, occ);
    DeviceBuf dtrace, dtc, dlen, drounds;
    const size_t ncount = (size_t)pl->dt.ncount;
    McArgs extra{};
    if (rc == HEA_OK) {
        if (dev_alloc(&drounds.p, count * sizeof(int64_t)) != cudaSuccess) rc = fail(HEA_ERR_NOMEM, "no memory");
        extra.rounds_out = (int64_t *)drounds.p;
        if (rc == HEA_OK && trace_cap > 0) {
            if (dev_alloc(&dtrace.p, (size_t)count * trace_cap * sizeof(AcceptRecord)) != cudaSuccess ||
                dev_alloc(&dlen.p, count * sizeof(int64_t)) != cudaSuccess ||
                (trace_counts &&
                 dev_alloc(&dtc.p, (size_t)count * trace_cap * ncount * sizeof(int32_t)) != cudaSuccess))
                rc = fail(HEA_ERR_NOMEM, "cannot allocate the trace buffers");
            extra.trace = (AcceptRecord *)dtrace.p;
            extra.trace_counts = (int32_t *)dtc.p;
            extra.trace_len = (int64_t *)dlen.p;
            extra.trace_cap = trace_cap;
        }
    }
    if (rc == HEA_OK) {
        cudaMemsetAsync(pl->stats, 0, 4 * sizeof(unsigned long long), pl->stream);
        rc = launch_mc(pl, pl->order, count, mc_call, extra);
    }
    if (rc == HEA_OK) rc = read_population(pl, count, occ, nullptr);
    auto copy = [&](void *dst, const void *src, size_t bytes) {
        if (rc != HEA_OK || !dst || !src) return;
        cudaError_t e = cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) rc = fail(HEA_ERR_CUDA, "copy failed: %s", cudaGetErrorString(e));
    };
    copy(out_counts, pl->cnt, (size_t)count * ncount * sizeof(int32_t));
    copy(out_f2, pl->f2, count * sizeof(double));
    copy(out_rounds, drounds.p, count * sizeof(int64_t));
    if (trace_cap > 0) {
        copy(trace, dtrace.p, (size_t)count * trace_cap * sizeof(AcceptRecord));
        copy(trace_len, dlen.p, count * sizeof(int64_t));
        copy(trace_counts, dtc.p, (size_t)count * trace_cap * ncount * sizeof(int32_t));
    }
    delete pl;
    return rc;
}

int hea_build_neighbors(int32_t lattice, int32_t cell, int32_t shell_set, int32_t *out_nbor, int32_t *out_shell_sizes,
                        int32_t *out_num_sites)
{
    if (cell < 1 || cell > 1024) return fail(HEA_ERR_INVALID, "cell must be 1..1024, got %d", cell);
    if (shell_set != 0 && shell_set != 1) return fail(HEA_ERR_INVALID, "shell_set must be 0 or 1");
    LatticeSpec sp;
    HEA_TRY(make_lattice_spec(lattice, shell_set, sp));
    const int64_t n = (int64_t)sp.nb * cell * cell * cell;
    if (n > INT32_MAX / 2) return fail(HEA_ERR_INVALID, "cell %d gives too many sites", cell);
    int row = 0;
    for (int k = 0; k < 3; ++k) {
        row += sp.size[k];
        if (out_shell_sizes) out_shell_sizes[k] = sp.size[k];
    }
    if (out_num_sites) *out_num_sites = (int32_t)n;
    if (!out_nbor) return HEA_OK;
    DeviceBuf d, derr;
    const size_t bytes = (size_t)n * row * sizeof(int32_t);
    if (dev_alloc(&d.p, bytes) != cudaSuccess || dev_alloc(&derr.p, sizeof(int)) != cudaSuccess)
        return fail(HEA_ERR_NOMEM, "cannot allocate %zu bytes for the neighbour table", bytes);
    HEA_CUDA(cudaMemset(derr.p, 0, sizeof(int)));
    const int blocks = (int)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096);
    build_neighbors_kernel<<<blocks, 256>>>(sp, cell, (int32_t *)d.p, row, (int *)derr.p);
    HEA_CUDA(cudaGetLastError());
    int herr = 0;
    HEA_CUDA(cudaMemcpy(&herr, derr.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (herr) return fail(HEA_ERR_INVALID, "lattice construction produced an off-lattice position");
    HEA_CUDA(cudaMemcpy(out_nbor, d.p, bytes, cudaMemcpyDeviceToHost));
    return HEA_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free recount (hea_recount_noalloc).
//
// For callers that cannot allocate device memory: processes whose device
// memory is fully reserved by another allocator (a framework's caching pool
// that claims the GPU at start-up), or code that must not pay cudaMalloc's
// implicit device-wide synchronisation.  Every device buffer the recount needs
// (raw and padded neighbour table, occupancy rows, slot order, counts, f2,
// error flag) is carved out of one fixed static array; nothing is allocated
// or freed.  The array is shared by all calls and keeps the previous call's
// contents: the error flag is cleared and the counts are rebuilt from zero on
// every call.  Two calls that overlap on the GPU (two host threads, or a call
// while another is still running) race on the array.
// ---------------------------------------------------------------------------
static __device__ __align__(256) unsigned char g_noalloc_scratch[HEA_NOALLOC_SCRATCH_BYTES];

namespace {

// Device address of the scratch array in the context current on this thread,
// looked up on every call: the address belongs to one context, so a cached one
// would be stale after a device reset or under another current context (a
// driver-API context on the same device), and the lookup costs far less than
// the call's synchronous copies.
int noalloc_scratch(void **out)
{
    void *p = nullptr;
    HEA_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    *out = p;
    return HEA_OK;
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

extern "C" int hea_recount_noalloc(const hea_problem *problem, int32_t count, const uint8_t *occ, int32_t *out_counts,
                                   double *out_f2)
{
    if (count < 1 || count > 65535) return fail(HEA_ERR_INVALID, "count must be 1..65535");
    if (!occ) return fail(HEA_ERR_INVALID, "occ is NULL");
    if (problem && !problem->nbor)
        return fail(HEA_ERR_UNSUPPORTED, "the allocation-free recount needs a neighbour table (nbor)");
    HEA_TRY(validate_problem(problem));
    const hea_problem *pb = problem;
    const int T = pb->num_types, S = pb->num_shells, N = pb->num_sites;
    const int ncount = S * T * T;

    // the recount's constants (fitness tables, padded shell geometry)
    SearchConst c;
    std::memset(&c, 0, sizeof(c));
    PadGeom g{};
    int raw_row = 0, poff = 0;
    for (int k = 0; k < S; ++k) {
        const int z = pb->shell_sizes[k], zp = (z + 3) & ~3;
        g.size[k] = z;
        g.off[k] = raw_row;
        g.poff[k] = poff;
        g.psize[k] = zp;
        c.off4[k] = poff / 4;
        c.chunks[k] = zp / 4;
        c.pad[k] = zp - z;
        raw_row += z;
        poff += zp;
    }
    g.num_shells = S;
    g.raw_row = raw_row;
    g.pad_row = poff;
    g.num_sites = N;
    c.row4 = poff / 4;
    c.num_sites = N;
    c.num_types = T;
    c.num_shells = S;
    c.occ_stride = (N + 15) & ~15;
    c.prefix[0] = 0;
    for (int t = 0; t < T; ++t) c.prefix[t + 1] = c.prefix[t] + pb->species[t];
    for (int k = 0; k < S; ++k) {
        c.w[k] = pb->weight[k];
        for (int i = 0; i < T; ++i)
            for (int j = 0; j < T; ++j) {
                const int e = (k * T + i) * T + j;
                c.E[e] = 1.0 - pb->target_sro[(size_t)k * T * T + i * T + j];
                c.R[e] = (double)N / (((double)pb->shell_sizes[k] * (double)pb->species[i]) * (double)pb->species[j]);
            }
    }
    // occupancies must hold the problem's composition
    for (int p = 0; p < count; ++p) {
        int64_t h[kMaxTypes] = {};
        for (int s = 0; s < N; ++s) {
            const uint8_t v = occ[(size_t)p * N + s];
            if (v >= T) return fail(HEA_ERR_INVALID, "occupancy holds species %d >= %d", v, T);
            ++h[v];
        }
        for (int t = 0; t < T; ++t)
            if (h[t] != c.prefix[t + 1] - c.prefix[t])
                return fail(HEA_ERR_INVALID, "occupancy %d has %lld atoms of species %d, element says %d", p,
                            (long long)h[t], t, c.prefix[t + 1] - c.prefix[t]);
    }

    // scratch layout
    const size_t raw_bytes = (size_t)N * raw_row * sizeof(int32_t);
    const size_t pad_bytes = (size_t)N * poff * sizeof(int32_t);
    const size_t o_raw = 0;
    const size_t o_pad = align256(o_raw + raw_bytes);
    const size_t o_occ = align256(o_pad + pad_bytes);
    const size_t o_cnt = align256(o_occ + (size_t)count * c.occ_stride);
    const size_t o_f2 = align256(o_cnt + (size_t)count * ncount * sizeof(int32_t));
    const size_t o_order = align256(o_f2 + (size_t)count * sizeof(double));
    const size_t o_err = align256(o_order + (size_t)count * sizeof(int32_t));
    const size_t need = o_err + sizeof(int);
    if (need > (size_t)HEA_NOALLOC_SCRATCH_BYTES)
        return fail(HEA_ERR_UNSUPPORTED,
                    "%d sites x %d occupancies need %zu bytes of scratch; the allocation-free recount has %zu "
                    "(HEA_NOALLOC_SCRATCH_BYTES)",
                    N, count, need, (size_t)HEA_NOALLOC_SCRATCH_BYTES);
    const size_t smem = (size_t)c.occ_stride + 16 + 4 * (size_t)((ncount + 3) & ~3);
    if (smem > (size_t)smem_limit())
        return fail(HEA_ERR_UNSUPPORTED, "%d sites need %zu bytes of shared memory, above the %d-byte limit", N, smem,
                    smem_limit());

    void *base = nullptr;
    HEA_TRY(noalloc_scratch(&base));
    unsigned char *sc = static_cast<unsigned char *>(base);
    int32_t *d_raw = reinterpret_cast<int32_t *>(sc + o_raw);
    int32_t *d_pad = reinterpret_cast<int32_t *>(sc + o_pad);
    uint8_t *d_occ = sc + o_occ;
    int32_t *d_cnt = reinterpret_cast<int32_t *>(sc + o_cnt);
    double *d_f2 = reinterpret_cast<double *>(sc + o_f2);
    int32_t *d_order = reinterpret_cast<int32_t *>(sc + o_order);
    int *d_err = reinterpret_cast<int *>(sc + o_err);

    const GenFn gen = kGen[T][S];
    HEA_CUDA(allow_max_smem(gen));
    HEA_CUDA(cudaMemcpy(d_raw, pb->nbor, raw_bytes, cudaMemcpyHostToDevice));
    HEA_CUDA(cudaMemset(d_err, 0, sizeof(int)));
    pad_and_check_kernel<<<1184, 256>>>(d_raw, d_pad, g, d_err);
    HEA_CUDA(cudaGetLastError());
    int herr = 0;
    HEA_CUDA(cudaMemcpy(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (herr & 1) return fail(HEA_ERR_INVALID, "neighbour list holds an id outside [0, %d)", N);
    if (herr & 2) return fail(HEA_ERR_UNSUPPORTED, "neighbour list names a site as its own neighbour");
    if (herr & 4) return fail(HEA_ERR_UNSUPPORTED, "neighbour list is not symmetric within a shell");
    HEA_CUDA(cudaMemcpy2D(d_occ, c.occ_stride, occ, N, N, count, cudaMemcpyHostToDevice));
    iota_kernel<<<(count + 255) / 256, 256>>>(d_order, count);
    HEA_CUDA(cudaGetLastError());
    GenArgs a{};
    a.nbor = reinterpret_cast<const int4 *>(d_pad);
    a.occ = d_occ;
    a.cnt = d_cnt;
    a.f2 = d_f2;
    a.order = d_order;
    a.generation = 0;
    a.generate = 0;
    gen<<<count, 512, smem>>>(c, a);
    HEA_CUDA(cudaGetLastError());
    // NULL outputs are skipped, as hea_recount skips them
    if (out_counts)
        HEA_CUDA(cudaMemcpy(out_counts, d_cnt, (size_t)count * ncount * sizeof(int32_t), cudaMemcpyDeviceToHost));
    if (out_f2) HEA_CUDA(cudaMemcpy(out_f2, d_f2, (size_t)count * sizeof(double), cudaMemcpyDeviceToHost));
    HEA_CUDA(cudaDeviceSynchronize());
    return HEA_OK;
}

// ---------------------------------------------------------------------------
// Batched search: many structures in one persistent kernel (hea_batch.cuh)
// ---------------------------------------------------------------------------
#include "hea_batch.cuh"

namespace {
struct BatchLevels {
    unsigned long long total[kBatchLevels], base[kBatchLevels];
};
}  // namespace
using BatchLevels_ = BatchLevels;

struct hea_batch {
    int count = 0;
    std::vector<DeviceTables *> tables;
    std::vector<BatchStruct> h_structs;
    std::vector<void *> buffers;  // every device allocation of the batch
    BatchStruct *d_structs = nullptr;
    BatchState *d_states = nullptr;
    BatchJob *d_jobs = nullptr;
    BatchCtl *d_ctl = nullptr;
    unsigned long long *d_finish = nullptr;  // per structure: ns from start to its last sort
    unsigned long long total_jobs = 0;
    size_t smem = 0;
    int grid = 0, block = HEA_BATCH_THREADS;
    cudaStream_t stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    uint8_t *out_occ = nullptr;
    double *out_f2 = nullptr;
    BatchLevels_ *lv = nullptr;  // queue layout of the graph's reset kernel
    int hbm_all = 1, ctas_per_sm = HEA_BATCH_MIN_BLOCKS;  // current launch configuration
    unsigned long long wait_limit_ns = 60ull * 1000000000ull;  // bound on every device-side wait
    ~hea_batch()
    {
        delete lv;
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        for (void *p : buffers) dev_free(p);  // back to the block cache
        for (DeviceTables *t : tables) delete t;
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

__global__ void batch_reset_kernel(BatchCtl *ctl, BatchJob *jobs, unsigned long long njobs, BatchLevels lv,
                                   unsigned long long limit_ns)
{
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < njobs;
         i += (unsigned long long)gridDim.x * blockDim.x)
        jobs[i].seq = 0;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        for (int l = 0; l < kBatchLevels; ++l) {
            ctl->q[l].head = 0;
            ctl->q[l].tail = 0;
            ctl->q[l].cap = lv.total[l] ? lv.total[l] : 1;
            ctl->q[l].base = lv.base[l];
        }
        for (int i = 0; i < 4; ++i) ctl->stats[i] = 0;
        ctl->error = 0;
        ctl->active = 0;
        ctl->wait_limit_ns = limit_ns;
        ctl->start_ns = global_ns();
        ctl->progress_ns = ctl->start_ns;
        ctl->deadline_ns = 0;
    }
}

template <class X>
int batch_alloc(hea_batch *b, X **p, size_t bytes)
{
    void *q = nullptr;  // from the block cache: a batch of the same shapes made again reuses the blocks
    if (dev_alloc(&q, bytes) != cudaSuccess) return fail(HEA_ERR_NOMEM, "cannot allocate %zu bytes", bytes);
    b->buffers.push_back(q);
    *p = static_cast<X *>(q);
    return HEA_OK;
}

int batch_layout(const SearchConst &c, int S)
{
    if (c.lat.L) return S == 1 ? kLayImp1 : (S == 2 ? kLayImp2 : kLayImp3);
    if (S == 3 && c.chunks[0] == 2 && c.chunks[1] == 2 && c.chunks[2] == 3) return kLayBcc;
    if (S == 3 && c.chunks[0] == 3 && c.chunks[1] == 2 && c.chunks[2] == 6) return kLayFccTrue;
    return S == 1 ? kLayRt1 : (S == 2 ? kLayRt2 : kLayRt3);
}

// Shared memory of one batch job: occupancy (unless it stays in HBM), then the
// search's delta table, swap records and count buffers.
size_t batch_job_smem(int occ_stride, int T, int S, int nwarps, bool hbm)
{
    return (hbm ? 0 : (size_t)occ_stride + 16) + search_smem_tail(T, S, nwarps);
}

// Dynamic shared memory per CTA that still lets HEA_BATCH_MIN_BLOCKS batch CTAs
// share an SM.
int batch_smem_budget(size_t *out, int ctas_per_sm = HEA_BATCH_MIN_BLOCKS)
{
    cudaFuncAttributes a;
    int dev = 0, per_sm = 0, reserved = 0;
    HEA_CUDA(cudaFuncGetAttributes(&a, batch_kernel));
    HEA_CUDA(cudaGetDevice(&dev));
    HEA_CUDA(cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
    HEA_CUDA(cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev));
    long long b = (long long)per_sm / ctas_per_sm - reserved - (long long)a.sharedSizeBytes;
    b &= ~127ll;
    const long long lim = (long long)smem_limit() - (long long)a.sharedSizeBytes;
    *out = (size_t)std::max(0ll, std::min(b, lim));
    return HEA_OK;
}

// Launch configuration of a batch: occupancy placement (hbm_all: every
// structure's occupancy in HBM; otherwise in shared memory where the per-CTA
// budget of ctas_per_sm CTAs per SM allows) and resident CTAs per SM; then the
// run is captured again as a CUDA graph.  Results do not depend on it.
int batch_configure(hea_batch *b, int hbm_all, int ctas_per_sm)
{
    const int nwarps = b->block / 32;
    size_t budget = 0;
    HEA_TRY(batch_smem_budget(&budget, ctas_per_sm));
    size_t smem = 0;
    for (int i = 0; i < b->count; ++i) {
        BatchStruct &d = b->h_structs[i];
        const int T = b->tables[i]->T, S = b->tables[i]->S;
        d.hbm = (hbm_all || batch_job_smem(d.c.occ_stride, T, S, nwarps, false) > budget) ? 1 : 0;
        smem = std::max(smem, batch_job_smem(d.c.occ_stride, T, S, nwarps, d.hbm != 0));
    }
    cudaFuncAttributes a;
    HEA_CUDA(cudaFuncGetAttributes(&a, batch_kernel));
    if (smem + a.sharedSizeBytes > (size_t)smem_limit())
        return fail(HEA_ERR_UNSUPPORTED, "the largest structure needs %zu bytes of shared memory, above %d", smem,
                    smem_limit() - (int)a.sharedSizeBytes);
    int per_sm = 0, sms = 0, dev = 0;
    HEA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_kernel, b->block, smem));
    HEA_CUDA(cudaGetDevice(&dev));
    HEA_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    per_sm = std::min(per_sm, ctas_per_sm);
    if (per_sm < 1) return fail(HEA_ERR_UNSUPPORTED, "batch kernel does not fit on an SM");
    b->smem = smem;
    b->grid = per_sm * sms;
    b->hbm_all = hbm_all;
    b->ctas_per_sm = per_sm;
    HEA_CUDA(cudaStreamSynchronize(b->stream));
    HEA_CUDA(cudaMemcpy(b->d_structs, b->h_structs.data(), sizeof(BatchStruct) * b->count, cudaMemcpyHostToDevice));
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    // the run as one CUDA graph: reset the queue, seed phase 0, persistent kernel
    HEA_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    batch_reset_kernel<<<64, 256, 0, b->stream>>>(b->d_ctl, b->d_jobs, b->total_jobs, *b->lv, b->wait_limit_ns);
    batch_seed_kernel<<<b->count, 256, 0, b->stream>>>(b->d_structs, nullptr, b->d_states, b->d_jobs, b->d_ctl);
    batch_kernel<<<b->grid, b->block, b->smem, b->stream>>>(b->d_structs, b->d_states, b->d_jobs, b->d_ctl,
                                                            b->d_finish);
    HEA_CUDA(cudaStreamEndCapture(b->stream, &b->graph));
    HEA_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
    return HEA_OK;
}

}  // namespace

extern "C" {

int hea_batch_create(const hea_problem *problems, const hea_params *params, int32_t count, hea_batch **out)
{
    if (!out) return fail(HEA_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (!problems || !params || count < 1) return fail(HEA_ERR_INVALID, "need at least one structure");
    hea_batch *b = new (std::nothrow) hea_batch();
    if (!b) return fail(HEA_ERR_NOMEM, "out of host memory");
    b->count = count;
    size_t hist_total = 0;  // site-histogram bytes of all structures (stream_histograms)
    for (int i = 0; i < count; ++i)
        hist_total += (size_t)2 * std::max(0, params[i].num_solutions) * std::max(0, problems[i].num_sites) *
                      sizeof(uint4);
    int rc = HEA_OK;
    for (int i = 0; i < count && rc == HEA_OK; ++i) {
        rc = validate_params(&params[i]);
        if (rc != HEA_OK) break;
        DeviceTables *t = new (std::nothrow) DeviceTables();
        if (!t) {
            rc = fail(HEA_ERR_NOMEM, "out of host memory");
            break;
        }
        b->tables.push_back(t);
        rc = build_tables(&problems[i], params[i].seed, *t);
        if (rc != HEA_OK) {
            std::string m = g_error;
            rc = fail(rc, "structure %d: %s", i, m.c_str());
            break;
        }
        const int P = params[i].num_solutions, slots = 2 * P;
        BatchStruct d{};
        d.c = t->c;
        d.c.hist_stream = stream_histograms((size_t)slots * t->N * sizeof(uint4), hist_total);
        d.nbor = t->nbor;
        d.P = P;
        d.Q = params[i].parallel_task;
        d.D = params[i].converge_depth;
        d.I = params[i].total_iter;
        d.max_rounds = params[i].max_rounds > 0 ? params[i].max_rounds : (int64_t)1 << 31;
        d.tol2 = -1.0;
        d.T = t->T;
        d.layout = batch_layout(t->c, t->S);
        if ((rc = batch_alloc(b, &d.occ, (size_t)slots * t->c.occ_stride)) != HEA_OK) break;
        if ((rc = batch_alloc(b, &d.cnt, (size_t)slots * t->ncount * sizeof(int32_t))) != HEA_OK) break;
        if ((rc = batch_alloc(b, &d.f2, (size_t)slots * sizeof(double))) != HEA_OK) break;
        if ((rc = batch_alloc(b, &d.order, (size_t)slots * sizeof(int32_t))) != HEA_OK) break;
        if ((rc = batch_alloc(b, &d.scratch, (size_t)slots * sizeof(int32_t))) != HEA_OK) break;
        if ((rc = batch_alloc(b, &d.hist, (size_t)slots * t->N * sizeof(uint4))) != HEA_OK) break;
        d.nbmask = t->nbmask;
        if (cudaMemset(d.occ, 0, (size_t)slots * t->c.occ_stride) != cudaSuccess) {
            rc = fail(HEA_ERR_CUDA, "cudaMemset failed");
            break;
        }
        b->h_structs.push_back(d);
        b->total_jobs += d.I > 0 ? (unsigned long long)P * (2 * d.I + 1) : (unsigned long long)P;
    }
    // priority levels: structures ranked by work, largest first
    BatchLevels lv{};
    if (rc == HEA_OK) {
        std::vector<int> rank(count);
        for (int i = 0; i < count; ++i) rank[i] = i;
        auto work = [&](int i) {
            const BatchStruct &d = b->h_structs[i];
            return (double)d.c.num_sites * d.P * (2.0 * d.I + 1.0);
        };
        std::stable_sort(rank.begin(), rank.end(), [&](int x, int y) { return work(x) > work(y); });
        for (int r = 0; r < count; ++r) {
            BatchStruct &d = b->h_structs[rank[r]];
            d.level = (int)((long long)r * kBatchLevels / count);
            lv.total[d.level] += d.I > 0 ? (unsigned long long)d.P * (2 * d.I + 1) : (unsigned long long)d.P;
        }
        for (int l = 1; l < kBatchLevels; ++l) lv.base[l] = lv.base[l - 1] + lv.total[l - 1];
    }
    size_t max_out = 0;
    for (int i = 0; rc == HEA_OK && i < count; ++i)
        max_out = std::max(max_out, (size_t)b->h_structs[i].P * b->h_structs[i].c.num_sites);
    if (rc == HEA_OK) rc = batch_alloc(b, &b->d_structs, sizeof(BatchStruct) * count);
    if (rc == HEA_OK) rc = batch_alloc(b, &b->d_states, sizeof(BatchState) * count);
    if (rc == HEA_OK) rc = batch_alloc(b, &b->d_jobs, sizeof(BatchJob) * b->total_jobs);
    if (rc == HEA_OK) rc = batch_alloc(b, &b->d_ctl, sizeof(BatchCtl));
    if (rc == HEA_OK) rc = batch_alloc(b, &b->d_finish, sizeof(unsigned long long) * count);
    if (rc == HEA_OK) rc = batch_alloc(b, &b->out_occ, max_out);
    if (rc == HEA_OK) rc = batch_alloc(b, &b->out_f2, sizeof(double) * 65536);
    if (rc == HEA_OK) {
        b->lv = new (std::nothrow) BatchLevels(lv);
        if (!b->lv) rc = fail(HEA_ERR_NOMEM, "out of host memory");
    }
    if (rc == HEA_OK) {
        cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreate(&b->ev0);
        if (e == cudaSuccess) e = cudaEventCreate(&b->ev1);
        if (e == cudaSuccess) e = allow_max_smem(batch_kernel);
        if (e != cudaSuccess) rc = fail(HEA_ERR_CUDA, "batch set-up failed: %s", cudaGetErrorString(e));
    }
    // Occupancy in HBM by default: with site-histogram scoring a search reads it
    // only for its draws, and small shared memory leaves room for more CTAs per
    // SM and a larger L1 (measured faster on the mixed batch; hea_batch_autotune
    // compares the alternatives on the batch at hand).
    if (rc == HEA_OK) rc = batch_configure(b, 1, HEA_BATCH_MIN_BLOCKS);
    if (rc != HEA_OK) {
        delete b;
        return rc;
    }
    *out = b;
    return HEA_OK;
}

int hea_batch_run(hea_batch *b, const uint64_t *seeds, hea_stats *stats)
{
    if (!b) return fail(HEA_ERR_INVALID, "batch is NULL");
    if (seeds) {
        for (int i = 0; i < b->count; ++i) {
            b->h_structs[i].c.key0 = (uint32_t)seeds[i];
            b->h_structs[i].c.key1 = (uint32_t)(seeds[i] >> 32);
        }
        HEA_CUDA(cudaMemcpyAsync(b->d_structs, b->h_structs.data(), sizeof(BatchStruct) * b->count,
                                 cudaMemcpyHostToDevice, b->stream));
    }
    HEA_CUDA(cudaEventRecord(b->ev0, b->stream));
    HEA_CUDA(cudaGraphLaunch(b->exec, b->stream));
    HEA_CUDA(cudaEventRecord(b->ev1, b->stream));
    HEA_CUDA(cudaStreamSynchronize(b->stream));
    BatchCtl ctl;
    HEA_CUDA(cudaMemcpy(&ctl, b->d_ctl, sizeof(ctl), cudaMemcpyDeviceToHost));
    if (ctl.error)
        return fail(HEA_ERR_CUDA, "batched search stopped: %s",
                    ctl.error == 2 ? "a job-ring slot was reused before it was read"
                                   : "a wait for queued work exceeded its time limit");
    if (ctl.stats[3] != (unsigned long long)b->count)
        return fail(HEA_ERR_CUDA, "batched search finished %llu of %d structures", ctl.stats[3], b->count);
    if (stats) {
        float ms = 0;
        HEA_CUDA(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
        stats->rounds = (int64_t)ctl.stats[0];
        stats->evals = (int64_t)ctl.stats[1];
        stats->accepts = (int64_t)ctl.stats[2];
        stats->gpu_ms = ms;
        stats->mc_ms = ms;
        stats->mc_launches = 1;
    }
    return HEA_OK;
}

int hea_batch_set_wait_limit(hea_batch *b, double ms)
{
    if (!b) return fail(HEA_ERR_INVALID, "batch is NULL");
    if (!(ms > 0.0) || ms > 3.6e6) return fail(HEA_ERR_INVALID, "wait limit must be in (0, 3600000] ms");
    b->wait_limit_ns = (unsigned long long)(ms * 1e6);
    return batch_configure(b, b->hbm_all, b->ctas_per_sm);  // the limit is a parameter of the captured reset
}

int hea_batch_autotune(hea_batch *b, int32_t *out_hbm_all, int32_t *out_ctas_per_sm)
{
    if (!b) return fail(HEA_ERR_INVALID, "batch is NULL");
    struct Cand {
        int hbm_all, ctas;
    };
    // occupancy in HBM or in shared memory where it fits, at the kernel's CTAs per SM or one fewer
    std::vector<Cand> cands;
    for (int hbm_all : {1, 0})
        for (int ctas : {HEA_BATCH_MIN_BLOCKS, HEA_BATCH_MIN_BLOCKS - 1})
            if (ctas >= 1) cands.push_back(Cand{hbm_all, ctas});
    double best_rate = -1.0;
    Cand best = cands[0];
    for (const Cand &cd : cands) {
        const int rc = batch_configure(b, cd.hbm_all, cd.ctas);
        if (rc == HEA_ERR_UNSUPPORTED) continue;  // this placement does not fit
        HEA_TRY(rc);
        hea_stats st{};
        HEA_TRY(hea_batch_run(b, nullptr, &st));  // warm-up
        HEA_TRY(hea_batch_run(b, nullptr, &st));
        const double rate = st.gpu_ms > 0 ? st.evals / st.gpu_ms : 0.0;
        if (rate > best_rate) {
            best_rate = rate;
            best = cd;
        }
    }
    HEA_TRY(batch_configure(b, best.hbm_all, best.ctas));
    if (out_hbm_all) *out_hbm_all = b->hbm_all;
    if (out_ctas_per_sm) *out_ctas_per_sm = b->ctas_per_sm;
    return HEA_OK;
}

int hea_batch_read(hea_batch *b, int32_t index, uint8_t *out_occ, double *out_fitness)
{
    if (!b || index < 0 || index >= b->count) return fail(HEA_ERR_INVALID, "no structure %d in the batch", index);
    const BatchStruct &d = b->h_structs[index];
    dim3 grid((d.c.num_sites + 255) / 256 < 64 ? (d.c.num_sites + 255) / 256 : 64, d.P);
    gather_rows_kernel<<<grid, 256, 0, b->stream>>>(d.occ, d.order, d.P, d.c.occ_stride, d.c.num_sites, d.f2,
                                                    b->out_occ, b->out_f2);
    HEA_CUDA(cudaGetLastError());
    if (out_occ)
        HEA_CUDA(cudaMemcpyAsync(out_occ, b->out_occ, (size_t)d.P * d.c.num_sites, cudaMemcpyDeviceToHost, b->stream));
    std::vector<double> f(d.P);
    HEA_CUDA(cudaMemcpyAsync(f.data(), b->out_f2, d.P * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
    HEA_CUDA(cudaStreamSynchronize(b->stream));
    if (out_fitness)
        for (int p = 0; p < d.P; ++p) out_fitness[p] = std::sqrt(f[p]);
    return HEA_OK;
}

int hea_batch_finish_times(hea_batch *b, double *out_ms)
{
    if (!b || !out_ms) return fail(HEA_ERR_INVALID, "batch and out_ms must not be NULL");
    std::vector<unsigned long long> ns(b->count);
    HEA_CUDA(cudaMemcpy(ns.data(), b->d_finish, sizeof(unsigned long long) * b->count, cudaMemcpyDeviceToHost));
    for (int i = 0; i < b->count; ++i) out_ms[i] = ns[i] * 1e-6;
    return HEA_OK;
}

int hea_batch_tallies(hea_batch *b, uint64_t *out)
{
    if (!b || !out) return fail(HEA_ERR_INVALID, "batch and out must not be NULL");
    std::vector<BatchState> st(b->count);
    HEA_CUDA(cudaMemcpy(st.data(), b->d_states, sizeof(BatchState) * b->count, cudaMemcpyDeviceToHost));
    for (int i = 0; i < b->count; ++i)
        for (int k = 0; k < 3; ++k) out[3 * i + k] = st[i].tally[k];
    return HEA_OK;
}

void hea_batch_destroy(hea_batch *b) { delete b; }

}  // extern "C"

// ---------------------------------------------------------------------------
// Serving loop (hea_server_*): the job engine of hea_batch.cuh run in time
// slices.  Between slices the host admits queued requests (tables built or
// uploaded into a device arena, phase-0 jobs seeded) and collects finished
// ones; requests still running keep their state on the device.
// ---------------------------------------------------------------------------
namespace {

using ServerClock = std::chrono::steady_clock;

// First-fit sub-allocation of one device buffer in 256-byte granules.
struct ArenaHeap {
    std::map<size_t, size_t> free_;  // offset -> bytes
    size_t total = 0, free_bytes = 0;
    static size_t round(size_t b) { return (b + 255) & ~(size_t)255; }
    void init(size_t bytes)
    {
        total = free_bytes = bytes & ~(size_t)255;
        free_.clear();
        if (total) free_[0] = total;
    }
    bool alloc(size_t bytes, size_t *off)
    {
        bytes = round(bytes);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < bytes) continue;
            *off = it->first;
            const size_t rest = it->second - bytes, next = it->first + bytes;
            free_.erase(it);
            if (rest) free_[next] = rest;
            free_bytes -= bytes;
            return true;
        }
        return false;
    }
    void release(size_t off, size_t bytes)
    {
        bytes = round(bytes);
        free_bytes += bytes;
        auto it = free_.emplace(off, bytes).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
};

struct ServerRequest {
    int64_t id = 0;
    int state = 0;  // 0 queued, 1 on the device, 2 finished, 3 failed
    hea_params params{};
    double tol2 = -1.0;
    int level = 0;
    int N = 0, T = 0, S = 0;
    std::vector<int32_t> shell_sizes, species, nbor;  // nbor empty for lattice requests
    std::vector<double> weight, target;
    int lattice = -1, cell = 0, shell_set = 0;
    int slot = -1, hbm = 0;
    size_t off = 0, bytes = 0;
    size_t hist_bytes = 0;  // site-histogram bytes of the placed request
    double t_submit = 0, t_admit = 0, t_finish = 0, device_ms = 0;
    int iterations = 0;
    unsigned long long tally[3] = {0, 0, 0};
    std::vector<uint8_t> occ;
    std::vector<double> fit;
    std::string error;

    hea_problem problem() const
    {
        hea_problem p{};
        p.num_sites = N;
        p.num_types = T;
        p.num_shells = S;
        p.shell_sizes = const_cast<int32_t *>(shell_sizes.data());
        p.nbor = nbor.empty() ? nullptr : const_cast<int32_t *>(nbor.data());
        p.species = const_cast<int32_t *>(species.data());
        p.weight = const_cast<double *>(weight.data());
        p.target_sro = const_cast<double *>(target.data());
        if (lattice >= 0) {  // lattice requests keep no table: neighbours from lattice arithmetic
            p.implicit_lattice = lattice + 1;
            p.lattice_cell = cell;
            p.lattice_shell_set = shell_set;
        }
        return p;
    }
};

// Arena bytes of a request: padded table, then 2P occupancy rows, counts,
// f2, order and sort scratch, each 256-byte aligned.
struct RequestLayout {
    size_t nbor, nbmask, hist, occ, cnt, f2, order, scratch, total;
};

RequestLayout request_layout(const SearchConst &c, int64_t pad_row, int S, int T, int P)
{
    RequestLayout L{};
    const size_t slots = 2 * (size_t)P;
    size_t o = 0;
    auto take = [&](size_t bytes) {
        const size_t at = o;
        o += ArenaHeap::round(bytes);
        return at;
    };
    L.nbor = take((size_t)c.num_sites * pad_row * sizeof(int32_t));
    L.nbmask = take(nbmask_words(c.num_sites) * sizeof(uint32_t));
    L.hist = take(slots * c.num_sites * sizeof(uint4));
    L.occ = take(slots * c.occ_stride);
    L.cnt = take(slots * (size_t)S * T * T * sizeof(int32_t));
    L.f2 = take(slots * sizeof(double));
    L.order = take(slots * sizeof(int32_t));
    L.scratch = take(slots * sizeof(int32_t));
    L.total = o;
    return L;
}

__global__ void server_arm_kernel(BatchCtl *ctl, unsigned long long slice_ns)
{
    const unsigned long long now = global_ns();
    ctl->deadline_ns = now + slice_ns;
    ctl->progress_ns = now;
}

}  // namespace

struct hea_server {
    hea_server_config cfg{};
    int nwarps = HEA_BATCH_THREADS / 32;
    int grid = 0;
    size_t smem = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::vector<void *> buffers;
    uint8_t *arena = nullptr;
    ArenaHeap heap;
    size_t hist_placed = 0;  // site-histogram bytes of the placed requests (stream_histograms)
    BatchStruct *d_structs = nullptr;
    BatchState *d_states = nullptr;
    BatchJob *d_jobs = nullptr;
    BatchCtl *d_ctl = nullptr;
    unsigned long long *d_finish = nullptr;
    int32_t *d_list = nullptr;
    int *d_err = nullptr;  // per slot: table check flags
    void *d_raw = nullptr;
    size_t raw_bytes = 0;
    void *d_out = nullptr;
    size_t out_bytes = 0;
    std::vector<BatchStruct> h_structs;
    BatchState *h_states = nullptr;          // pinned: slice results, copied while the host works
    unsigned long long *h_finish = nullptr;  // pinned
    BatchCtl *h_ctl = nullptr;               // pinned
    uint8_t *h_stage = nullptr;              // pinned staging of finished populations
    size_t stage_bytes = 0;
    cudaStream_t side = nullptr;             // copies of finished populations
    cudaEvent_t ev_gather = nullptr;
    bool inflight = false;                   // a slice was launched and not yet waited for
    std::vector<int64_t> finished_ids;       // finished, not yet taken by hea_server_take_finished
    std::vector<int> h_err;
    std::vector<int32_t> h_list;
    std::vector<int64_t> slot_req;                // request id per slot, 0 = free
    unsigned long long level_load[kBatchLevels] = {};  // ring slots held per level
    std::map<int64_t, ServerRequest> reqs;
    std::deque<int64_t> queue;
    int64_t next_id = 1;
    ServerClock::time_point t0;
    double busy_ms = 0;
    int launches = 0;
    int running = 0;
    unsigned long long finished_total = 0;
    BatchCtl last_ctl{};
    std::string broken;  // set after a device-side failure; every later call fails with it

    ~hea_server()
    {
        if (stream) cudaStreamSynchronize(stream);
        if (side) cudaStreamSynchronize(side);
        for (void *p : buffers) cudaFree(p);
        if (d_raw) cudaFree(d_raw);
        if (d_out) cudaFree(d_out);
        for (void *p : {(void *)h_states, (void *)h_finish, (void *)h_ctl, (void *)h_stage})
            if (p) cudaFreeHost(p);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (ev_gather) cudaEventDestroy(ev_gather);
        if (side) cudaStreamDestroy(side);
        if (stream) cudaStreamDestroy(stream);
    }
    double now_ms() const
    {
        return std::chrono::duration<double, std::milli>(ServerClock::now() - t0).count();
    }
    template <class X>
    int alloc(X **p, size_t bytes)
    {
        void *q = nullptr;
        if (cudaMalloc(&q, bytes) != cudaSuccess) return fail(HEA_ERR_NOMEM, "cannot allocate %zu bytes", bytes);
        buffers.push_back(q);
        *p = static_cast<X *>(q);
        return HEA_OK;
    }
    // grow a scratch buffer between slices (nothing of this server is running)
    int grow(void **p, size_t *have, size_t need)
    {
        if (need <= *have) return HEA_OK;
        HEA_CUDA(cudaStreamSynchronize(stream));
        HEA_CUDA(cudaStreamSynchronize(side));
        if (*p) cudaFree(*p);
        *p = nullptr;
        *have = 0;
        if (cudaMalloc(p, need) != cudaSuccess) return fail(HEA_ERR_NOMEM, "cannot allocate %zu bytes", need);
        *have = need;
        return HEA_OK;
    }
};

namespace {

int server_broken(hea_server *sv) { return fail(HEA_ERR_CUDA, "server stopped: %s", sv->broken.c_str()); }

// Arena layout, table preparation and structure entry of one request in
// `slot`.  Returns HEA_OK, or HEA_PENDING when memory or ring room is short
// (the request stays queued).
int server_place(hea_server *sv, ServerRequest &r, int slot)
{
    const hea_problem pb = r.problem();
    SearchConst c;
    PadGeom g;
    fill_const(&pb, r.params.seed, c, g);
    const bool implicit = c.lat.L > 0;  // lattice requests: no table in the arena
    const int P = r.params.num_solutions;
    const RequestLayout L = request_layout(c, implicit ? 0 : g.pad_row, r.S, r.T, P);
    if (sv->level_load[r.level] + 2ull * P > (unsigned long long)sv->cfg.ring_jobs) return HEA_PENDING;
    size_t off = 0;
    if (!sv->heap.alloc(L.total, &off)) return HEA_PENDING;
    r.off = off;
    r.bytes = L.total;
    uint8_t *base = sv->arena + off;

    // uploaded tables: the raw table, then its padded, checked copy; lattice requests: nothing
    cudaError_t e = cudaMemsetAsync(sv->d_err + slot, 0, sizeof(int), sv->stream);
    if (!implicit) {
        const size_t raw = (size_t)r.N * g.raw_row * sizeof(int32_t);
        int rc = sv->grow(&sv->d_raw, &sv->raw_bytes, raw);
        if (rc != HEA_OK) {
            sv->heap.release(off, L.total);
            return rc;
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(sv->d_raw, r.nbor.data(), raw, cudaMemcpyHostToDevice, sv->stream);
        if (e == cudaSuccess) {
            pad_and_check_kernel<<<1184, 256, 0, sv->stream>>>((const int32_t *)sv->d_raw,
                                                                (int32_t *)(base + L.nbor), g, sv->d_err + slot);
            e = cudaGetLastError();
        }
    }
    if (e == cudaSuccess) e = cudaMemsetAsync(base + L.nbmask, 0, L.hist - L.nbmask, sv->stream);
    if (e == cudaSuccess) {
        if (implicit)
            nbmask_implicit_kernel<<<1184, 256, 0, sv->stream>>>(c, implicit_row(c, r.S),
                                                                  (uint32_t *)(base + L.nbmask));
        else
            nbmask_kernel<<<1184, 256, 0, sv->stream>>>((const int32_t *)(base + L.nbor), r.N, g.pad_row,
                                                         (uint32_t *)(base + L.nbmask));
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemsetAsync(base + L.occ, 0, L.cnt - L.occ, sv->stream);
    if (e != cudaSuccess) {
        sv->heap.release(off, L.total);
        return fail(HEA_ERR_CUDA, "request set-up failed: %s", cudaGetErrorString(e));
    }
    BatchStruct d{};
    d.c = c;
    r.hist_bytes = (size_t)2 * P * r.N * sizeof(uint4);
    sv->hist_placed += r.hist_bytes;
    d.c.hist_stream = stream_histograms(r.hist_bytes, sv->hist_placed);
    d.nbor = implicit ? nullptr : reinterpret_cast<const int4 *>(base + L.nbor);
    d.occ = base + L.occ;
    d.cnt = reinterpret_cast<int32_t *>(base + L.cnt);
    d.f2 = reinterpret_cast<double *>(base + L.f2);
    d.order = reinterpret_cast<int32_t *>(base + L.order);
    d.scratch = reinterpret_cast<int32_t *>(base + L.scratch);
    d.hist = reinterpret_cast<uint4 *>(base + L.hist);
    d.nbmask = reinterpret_cast<const uint32_t *>(base + L.nbmask);
    d.P = P;
    d.Q = r.params.parallel_task;
    d.D = r.params.converge_depth;
    d.I = r.params.total_iter;
    d.max_rounds = r.params.max_rounds > 0 ? r.params.max_rounds : (int64_t)1 << 31;
    d.tol2 = r.tol2;
    d.T = r.T;
    d.layout = batch_layout(c, r.S);
    d.level = r.level;
    d.hbm = (batch_job_smem(c.occ_stride, r.T, r.S, sv->nwarps, false) > sv->smem ||
             sv->cfg.hbm_sites == 0 || (sv->cfg.hbm_sites > 0 && r.N >= sv->cfg.hbm_sites))
                ? 1
                : 0;
    r.hbm = d.hbm;
    sv->h_structs[slot] = d;
    sv->level_load[r.level] += 2ull * P;
    r.slot = slot;
    return HEA_OK;
}

void server_release(hea_server *sv, ServerRequest &r)
{
    if (r.slot < 0) return;
    sv->heap.release(r.off, r.bytes);
    sv->hist_placed -= r.hist_bytes;
    sv->level_load[r.level] -= 2ull * r.params.num_solutions;
    sv->slot_req[r.slot] = 0;
    r.slot = -1;
}

// Admit queued requests in submission order while slots, arena memory and
// ring room allow; seed their phase-0 jobs.
int server_admit(hea_server *sv)
{
    std::vector<int64_t> placed;
    while (!sv->queue.empty()) {
        int slot = -1;
        for (int i = 0; i < sv->cfg.max_requests; ++i)
            if (sv->slot_req[i] == 0) {
                slot = i;
                break;
            }
        if (slot < 0) break;
        ServerRequest &r = sv->reqs[sv->queue.front()];
        const int rc = server_place(sv, r, slot);
        if (rc == HEA_PENDING) break;
        if (rc != HEA_OK) return rc;
        sv->slot_req[slot] = r.id;
        placed.push_back(r.id);
        sv->queue.pop_front();
    }
    if (placed.empty()) return HEA_OK;
    // table checks of the placed requests
    HEA_CUDA(cudaMemcpyAsync(sv->h_err.data(), sv->d_err, sizeof(int) * sv->cfg.max_requests, cudaMemcpyDeviceToHost,
                             sv->stream));
    HEA_CUDA(cudaStreamSynchronize(sv->stream));
    sv->h_list.clear();
    const double t = sv->now_ms();
    for (int64_t id : placed) {
        ServerRequest &r = sv->reqs[id];
        const int err = sv->h_err[r.slot];
        if (err) {
            r.state = 3;
            r.error = (err & 1) ? "neighbour list holds an id outside the structure"
                      : (err & 2) ? "neighbour list names a site as its own neighbour"
                                  : "neighbour list is not symmetric within a shell";
            r.t_finish = t;
            server_release(sv, r);
            sv->finished_ids.push_back(id);
            continue;
        }
        r.state = 1;
        r.t_admit = t;
        sv->h_list.push_back(r.slot);
        HEA_CUDA(cudaMemcpyAsync(sv->d_structs + r.slot, &sv->h_structs[r.slot], sizeof(BatchStruct),
                                 cudaMemcpyHostToDevice, sv->stream));
        ++sv->running;
    }
    if (sv->h_list.empty()) return HEA_OK;
    HEA_CUDA(cudaMemcpyAsync(sv->d_list, sv->h_list.data(), sizeof(int32_t) * sv->h_list.size(),
                             cudaMemcpyHostToDevice, sv->stream));
    batch_seed_kernel<<<(unsigned)sv->h_list.size(), 256, 0, sv->stream>>>(sv->d_structs, sv->d_list, sv->d_states,
                                                                             sv->d_jobs, sv->d_ctl);
    HEA_CUDA(cudaGetLastError());
    return HEA_OK;
}

// Requests that finished in the last slice leave the device: their
// populations are gathered on the server stream (the GPU is idle between
// slices), the device copy to pinned staging runs on the side stream while the
// next slice computes, and their slots and arena memory are released at once
// (later work on the server stream is ordered after the gathers).
struct Collect {
    int64_t id;
    size_t off, off_f2;
    int P, N;
};

int server_collect_start(hea_server *sv, std::vector<Collect> &col)
{
    const double t = sv->now_ms();
    size_t total = 0;
    for (int slot = 0; slot < sv->cfg.max_requests; ++slot) {
        const int64_t id = sv->slot_req[slot];
        if (!id || !sv->h_states[slot].done) continue;
        ServerRequest &r = sv->reqs[id];
        if (r.state != 1) continue;
        const BatchStruct &d = sv->h_structs[slot];
        Collect c{id, total, 0, d.P, d.c.num_sites};
        total += ((size_t)d.P * d.c.num_sites + 7) & ~(size_t)7;
        c.off_f2 = total;
        total += (size_t)d.P * sizeof(double);
        col.push_back(c);
        r.t_finish = t;
        r.device_ms = sv->h_finish[slot] * 1e-6;
        r.iterations = sv->h_states[slot].phase;
        for (int k = 0; k < 3; ++k) r.tally[k] = sv->h_states[slot].tally[k];
    }
    if (col.empty()) return HEA_OK;
    HEA_TRY(sv->grow(&sv->d_out, &sv->out_bytes, total));
    if (total > sv->stage_bytes) {
        if (sv->h_stage) cudaFreeHost(sv->h_stage);
        sv->h_stage = nullptr;
        sv->stage_bytes = 0;
        if (cudaMallocHost((void **)&sv->h_stage, total) != cudaSuccess)
            return fail(HEA_ERR_NOMEM, "cannot allocate %zu bytes of pinned staging", total);
        sv->stage_bytes = total;
    }
    uint8_t *out = (uint8_t *)sv->d_out;
    for (const Collect &c : col) {
        ServerRequest &r = sv->reqs[c.id];
        const BatchStruct &d = sv->h_structs[r.slot];
        dim3 grid((unsigned)std::min(64, (c.N + 255) / 256), (unsigned)c.P);
        gather_rows_kernel<<<grid, 256, 0, sv->stream>>>(d.occ, d.order, c.P, d.c.occ_stride, c.N, d.f2, out + c.off,
                                                        reinterpret_cast<double *>(out + c.off_f2));
        HEA_CUDA(cudaGetLastError());
        server_release(sv, r);
        --sv->running;
    }
    HEA_CUDA(cudaEventRecord(sv->ev_gather, sv->stream));
    HEA_CUDA(cudaStreamWaitEvent(sv->side, sv->ev_gather, 0));
    HEA_CUDA(cudaMemcpyAsync(sv->h_stage, sv->d_out, total, cudaMemcpyDeviceToHost, sv->side));
    return HEA_OK;
}

int server_collect_finish(hea_server *sv, const std::vector<Collect> &col, int32_t *finished)
{
    if (col.empty()) return HEA_OK;
    HEA_CUDA(cudaStreamSynchronize(sv->side));
    for (const Collect &c : col) {
        ServerRequest &r = sv->reqs[c.id];
        r.occ.assign(sv->h_stage + c.off, sv->h_stage + c.off + (size_t)c.P * c.N);
        r.fit.resize(c.P);
        std::memcpy(r.fit.data(), sv->h_stage + c.off_f2, c.P * sizeof(double));
        for (double &f : r.fit) f = std::sqrt(f);
        r.state = 2;
        sv->finished_ids.push_back(c.id);
        ++sv->finished_total;
        ++*finished;
    }
    return HEA_OK;
}

void fill_info(const ServerRequest &r, hea_request_info *info)
{
    if (!info) return;
    std::memset(info, 0, sizeof(*info));
    info->state = r.state;
    info->iterations = r.iterations;
    info->hbm = r.hbm;
    info->submit_ms = r.t_submit;
    info->admit_ms = r.t_admit;
    info->finish_ms = r.t_finish;
    info->device_ms = r.device_ms;
    info->rounds = (int64_t)r.tally[0];
    info->evals = (int64_t)r.tally[1];
    info->accepts = (int64_t)r.tally[2];
    info->device_bytes = (int64_t)r.bytes;
}

int server_enqueue(hea_server *sv, ServerRequest &&r, const hea_params *params, double tolerance, int32_t priority,
                   int64_t *out_id)
{
    HEA_TRY(validate_params(params));
    if (std::isnan(tolerance) || tolerance == INFINITY) return fail(HEA_ERR_INVALID, "tolerance must be finite");
    if (priority < 0 || priority >= kBatchLevels)
        return fail(HEA_ERR_INVALID, "priority must be 0..%d, got %d", kBatchLevels - 1, priority);
    if (params->max_rounds > ((int64_t)1 << 31))
        return fail(HEA_ERR_INVALID, "max_rounds above 2^31 is not supported by the server");
    if (2ll * params->num_solutions > sv->cfg.ring_jobs)
        return fail(HEA_ERR_UNSUPPORTED, "2 * nnet = %d exceeds the job ring (%d)", 2 * params->num_solutions,
                    sv->cfg.ring_jobs);
    r.params = *params;
    r.tol2 = tolerance >= 0 ? tolerance * tolerance : -1.0;
    r.level = priority;
    {  // memory the request will need must fit the arena at all
        const hea_problem pb = r.problem();
        SearchConst c;
        PadGeom g;
        fill_const(&pb, params->seed, c, g);
        const RequestLayout L = request_layout(c, c.lat.L ? 0 : g.pad_row, r.S, r.T, params->num_solutions);
        if (L.total > sv->heap.total)
            return fail(HEA_ERR_UNSUPPORTED, "request needs %zu bytes of device memory; the arena holds %zu", L.total,
                        sv->heap.total);
    }
    r.id = sv->next_id++;
    r.state = 0;
    r.t_submit = sv->now_ms();
    const int64_t id = r.id;
    sv->reqs.emplace(id, std::move(r));
    sv->queue.push_back(id);
    if (out_id) *out_id = id;
    return HEA_OK;
}

}  // namespace

extern "C" {

int hea_server_create(const hea_server_config *config, hea_server **out)
{
    if (!out) return fail(HEA_ERR_INVALID, "out is NULL");
    *out = nullptr;
    hea_server_config cfg{};
    if (config) cfg = *config;
    if (cfg.max_requests <= 0) cfg.max_requests = 256;
    if (cfg.ring_jobs <= 0) cfg.ring_jobs = 65536;
    if (cfg.slice_ms <= 0) cfg.slice_ms = 20.0;
    if (cfg.wait_limit_ms <= 0) cfg.wait_limit_ms = 10000.0;
    if (cfg.wait_limit_ms > 3.6e6) return fail(HEA_ERR_INVALID, "wait_limit_ms must be <= 3600000");
    if (cfg.max_requests > 65536) return fail(HEA_ERR_INVALID, "max_requests must be <= 65536");
    if (cfg.ring_jobs > (1 << 26)) return fail(HEA_ERR_INVALID, "ring_jobs must be <= 2^26");
    hea_server *sv = new (std::nothrow) hea_server();
    if (!sv) return fail(HEA_ERR_NOMEM, "out of host memory");
    sv->t0 = ServerClock::now();
    int rc = HEA_OK;
    if (cfg.arena_bytes <= 0) {
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) rc = fail(HEA_ERR_CUDA, "cannot query device memory");
        cfg.arena_bytes = (int64_t)std::min(fr / 2, (size_t)8 << 30);
    }
    size_t budget = 0;
    if (rc == HEA_OK) rc = batch_smem_budget(&budget);
    if (rc == HEA_OK) {
        const size_t least = batch_job_smem(0, kMaxTypes, kMaxShells, sv->nwarps, true);
        sv->smem = cfg.smem_bytes > 0 ? (size_t)cfg.smem_bytes : (cfg.hbm_sites == 0 ? least : budget);
        sv->smem = std::max(sv->smem, least);
        cudaFuncAttributes a;
        if (cudaFuncGetAttributes(&a, batch_kernel) != cudaSuccess) rc = fail(HEA_ERR_CUDA, "cannot query the batch kernel");
        else if (sv->smem + a.sharedSizeBytes > (size_t)smem_limit())
            rc = fail(HEA_ERR_INVALID, "smem_bytes %zu above the device limit", sv->smem);
        cfg.smem_bytes = (int32_t)sv->smem;
    }
    sv->cfg = cfg;
    const int M = cfg.max_requests;
    if (rc == HEA_OK) rc = sv->alloc(&sv->arena, (size_t)cfg.arena_bytes);
    if (rc == HEA_OK) rc = sv->alloc(&sv->d_structs, sizeof(BatchStruct) * M);
    if (rc == HEA_OK) rc = sv->alloc(&sv->d_states, sizeof(BatchState) * M);
    if (rc == HEA_OK) rc = sv->alloc(&sv->d_jobs, sizeof(BatchJob) * (size_t)cfg.ring_jobs * kBatchLevels);
    if (rc == HEA_OK) rc = sv->alloc(&sv->d_ctl, sizeof(BatchCtl));
    if (rc == HEA_OK) rc = sv->alloc(&sv->d_finish, sizeof(unsigned long long) * M);
    if (rc == HEA_OK) rc = sv->alloc(&sv->d_list, sizeof(int32_t) * M);
    if (rc == HEA_OK) rc = sv->alloc(&sv->d_err, sizeof(int) * M);
    if (rc == HEA_OK) {
        sv->heap.init((size_t)cfg.arena_bytes);
        sv->h_structs.assign(M, BatchStruct{});
        sv->h_err.assign(M, 0);
        sv->slot_req.assign(M, 0);
        sv->h_list.reserve(M);
        cudaError_t e = allow_max_smem(batch_kernel);
        int per_sm = 0, sms = 0, dev = 0;
        if (e == cudaSuccess)
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_kernel, HEA_BATCH_THREADS, sv->smem);
        if (e == cudaSuccess) e = cudaGetDevice(&dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e == cudaSuccess) e = cudaMallocHost((void **)&sv->h_states, sizeof(BatchState) * M);
        if (e == cudaSuccess) e = cudaMallocHost((void **)&sv->h_finish, sizeof(unsigned long long) * M);
        if (e == cudaSuccess) e = cudaMallocHost((void **)&sv->h_ctl, sizeof(BatchCtl));
        if (e == cudaSuccess) {
            std::memset(sv->h_states, 0, sizeof(BatchState) * M);
            std::memset(sv->h_finish, 0, sizeof(unsigned long long) * M);
            std::memset(sv->h_ctl, 0, sizeof(BatchCtl));
        }
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&sv->stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&sv->side, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sv->ev_gather, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreate(&sv->ev0);
        if (e == cudaSuccess) e = cudaEventCreate(&sv->ev1);
        if (e == cudaSuccess) e = cudaMemsetAsync(sv->d_states, 0, sizeof(BatchState) * M, sv->stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(sv->d_finish, 0, sizeof(unsigned long long) * M, sv->stream);
        if (e == cudaSuccess) {
            BatchLevels lv{};
            for (int l = 0; l < kBatchLevels; ++l) {
                lv.total[l] = (unsigned long long)cfg.ring_jobs;
                lv.base[l] = (unsigned long long)l * cfg.ring_jobs;
            }
            batch_reset_kernel<<<64, 256, 0, sv->stream>>>(sv->d_ctl, sv->d_jobs,
                                                          (unsigned long long)cfg.ring_jobs * kBatchLevels, lv,
                                                          (unsigned long long)(cfg.wait_limit_ms * 1e6));
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(sv->stream);
        if (e != cudaSuccess) rc = fail(HEA_ERR_CUDA, "server set-up failed: %s", cudaGetErrorString(e));
        else if (per_sm < 1) rc = fail(HEA_ERR_UNSUPPORTED, "batch kernel does not fit on an SM");
        sv->grid = per_sm * sms;
    }
    if (rc != HEA_OK) {
        delete sv;
        return rc;
    }
    *out = sv;
    return HEA_OK;
}

int hea_server_submit(hea_server *server, const hea_problem *problem, const hea_params *params, double tolerance,
                      int32_t priority, int64_t *out_id)
{
    if (!server) return fail(HEA_ERR_INVALID, "server is NULL");
    if (!server->broken.empty()) return server_broken(server);
    HEA_TRY(validate_problem(problem));
    ServerRequest r;
    r.N = problem->num_sites;
    r.T = problem->num_types;
    r.S = problem->num_shells;
    r.shell_sizes.assign(problem->shell_sizes, problem->shell_sizes + r.S);
    r.species.assign(problem->species, problem->species + r.T);
    r.weight.assign(problem->weight, problem->weight + r.S);
    r.target.assign(problem->target_sro, problem->target_sro + (size_t)r.S * r.T * r.T);
    int code = 0, cell = 0, shell_set = 0;
    if (problem->nbor && lattice_candidate(problem, code, cell, shell_set) &&
        table_is_lattice(problem, code, cell, shell_set)) {
        // an FCC/BCC cube's table: the request runs on lattice arithmetic, as a lattice request
        r.lattice = code - 1;
        r.cell = cell;
        r.shell_set = shell_set;
    } else if (problem->nbor) {
        int64_t row = 0;
        for (int k = 0; k < r.S; ++k) row += r.shell_sizes[k];
        r.nbor.assign(problem->nbor, problem->nbor + (size_t)r.N * row);
    } else {  // implicit neighbours: the request keeps its lattice, no table
        r.lattice = problem->implicit_lattice - 1;
        r.cell = problem->lattice_cell;
        r.shell_set = problem->lattice_shell_set;
    }
    return server_enqueue(server, std::move(r), params, tolerance, priority, out_id);
}

int hea_server_submit_lattice(hea_server *server, int32_t lattice, int32_t cell, int32_t shell_set,
                              int32_t num_types, int32_t num_shells, const int32_t *species, const double *weight,
                              const double *target_sro, const hea_params *params, double tolerance,
                              int32_t priority, int64_t *out_id)
{
    if (!server) return fail(HEA_ERR_INVALID, "server is NULL");
    if (!server->broken.empty()) return server_broken(server);
    int32_t sizes[3] = {0, 0, 0}, n = 0;
    HEA_TRY(hea_build_neighbors(lattice, cell, shell_set, nullptr, sizes, &n));
    if (num_shells < 1 || num_shells > 3) return fail(HEA_ERR_UNSUPPORTED, "num_shells must be 1..3, got %d", num_shells);
    if (!species || !weight || !target_sro) return fail(HEA_ERR_INVALID, "species, weight and target_sro are required");
    ServerRequest r;
    r.N = n;
    r.T = num_types;
    r.S = num_shells;
    r.shell_sizes.assign(sizes, sizes + num_shells);
    if (num_types < 1 || num_types > kMaxTypes)
        return fail(HEA_ERR_UNSUPPORTED, "number of species must be 2..%d, got %d", kMaxTypes, num_types);
    r.species.assign(species, species + num_types);
    r.weight.assign(weight, weight + num_shells);
    r.target.assign(target_sro, target_sro + (size_t)num_shells * num_types * num_types);
    r.lattice = lattice;
    r.cell = cell;
    r.shell_set = shell_set;
    const hea_problem pb = r.problem();
    HEA_TRY(validate_problem(&pb, false));
    return server_enqueue(server, std::move(r), params, tolerance, priority, out_id);
}

int hea_server_step(hea_server *server, int32_t *out_finished)
{
    if (!server) return fail(HEA_ERR_INVALID, "server is NULL");
    if (out_finished) *out_finished = 0;
    hea_server *sv = server;
    if (!sv->broken.empty()) return server_broken(sv);
    const int M = sv->cfg.max_requests;
    // 1. the previous slice: wait for it and its state copies
    if (sv->inflight) {
        HEA_CUDA(cudaStreamSynchronize(sv->stream));
        sv->inflight = false;
        float ms = 0;
        HEA_CUDA(cudaEventElapsedTime(&ms, sv->ev0, sv->ev1));
        sv->busy_ms += ms;
        ++sv->launches;
        sv->last_ctl = *sv->h_ctl;
        if (sv->last_ctl.error) {
            sv->broken = sv->last_ctl.error == 2 ? "a job-ring slot was reused before it was read"
                                                 : "a wait for queued work exceeded its time limit";
            return server_broken(sv);
        }
    }
    // 2. finished requests: gather, release, copy out behind the next slice
    std::vector<Collect> col;
    HEA_TRY(server_collect_start(sv, col));
    // 3. admission, then the next slice
    HEA_TRY(server_admit(sv));
    if (sv->running > 0) {
        HEA_CUDA(cudaEventRecord(sv->ev0, sv->stream));
        server_arm_kernel<<<1, 1, 0, sv->stream>>>(sv->d_ctl, (unsigned long long)(sv->cfg.slice_ms * 1e6));
        batch_kernel<<<sv->grid, HEA_BATCH_THREADS, sv->smem, sv->stream>>>(sv->d_structs, sv->d_states,
                                                                             sv->d_jobs, sv->d_ctl, sv->d_finish);
        HEA_CUDA(cudaGetLastError());
        HEA_CUDA(cudaEventRecord(sv->ev1, sv->stream));
        HEA_CUDA(cudaMemcpyAsync(sv->h_ctl, sv->d_ctl, sizeof(BatchCtl), cudaMemcpyDeviceToHost, sv->stream));
        HEA_CUDA(cudaMemcpyAsync(sv->h_states, sv->d_states, sizeof(BatchState) * M, cudaMemcpyDeviceToHost,
                                 sv->stream));
        HEA_CUDA(cudaMemcpyAsync(sv->h_finish, sv->d_finish, sizeof(unsigned long long) * M,
                                 cudaMemcpyDeviceToHost, sv->stream));
        sv->inflight = true;
    }
    // 4. hand the finished populations over while the slice runs
    int32_t fin = 0;
    HEA_TRY(server_collect_finish(sv, col, &fin));
    if (out_finished) *out_finished = fin;
    return HEA_OK;
}

int hea_server_take_finished(hea_server *server, int64_t *ids, int32_t cap, int32_t *count)
{
    if (!server || !count || (cap > 0 && !ids)) return fail(HEA_ERR_INVALID, "server, ids and count are required");
    const int32_t n = (int32_t)std::min<size_t>(server->finished_ids.size(), cap > 0 ? (size_t)cap : 0);
    for (int32_t i = 0; i < n; ++i) ids[i] = server->finished_ids[i];
    server->finished_ids.erase(server->finished_ids.begin(), server->finished_ids.begin() + n);
    *count = n;
    return HEA_OK;
}

int hea_server_info(hea_server *server, int64_t id, hea_request_info *info)
{
    if (!server) return fail(HEA_ERR_INVALID, "server is NULL");
    auto it = server->reqs.find(id);
    if (it == server->reqs.end()) return fail(HEA_ERR_INVALID, "no request %lld", (long long)id);
    fill_info(it->second, info);
    return HEA_OK;
}

int hea_server_result(hea_server *server, int64_t id, uint8_t *out_occ, double *out_fitness, hea_request_info *info)
{
    if (!server) return fail(HEA_ERR_INVALID, "server is NULL");
    auto it = server->reqs.find(id);
    if (it == server->reqs.end()) return fail(HEA_ERR_INVALID, "no request %lld", (long long)id);
    ServerRequest &r = it->second;
    fill_info(r, info);
    if (r.state == 0 || r.state == 1) return HEA_PENDING;
    if (r.state == 3) {
        const std::string m = r.error;
        server->reqs.erase(it);
        return fail(HEA_ERR_UNSUPPORTED, "request %lld failed: %s", (long long)id, m.c_str());
    }
    if (out_occ) std::memcpy(out_occ, r.occ.data(), r.occ.size());
    if (out_fitness) std::memcpy(out_fitness, r.fit.data(), r.fit.size() * sizeof(double));
    server->reqs.erase(it);
    return HEA_OK;
}

int hea_server_status_get(hea_server *server, hea_server_status *status)
{
    if (!server || !status) return fail(HEA_ERR_INVALID, "server and status must not be NULL");
    std::memset(status, 0, sizeof(*status));
    int unread = 0, free_slots = 0;
    for (const auto &kv : server->reqs) unread += (kv.second.state == 2 || kv.second.state == 3);
    for (int64_t s : server->slot_req) free_slots += (s == 0);
    status->queued = (int32_t)server->queue.size();
    status->running = server->running;
    status->finished_unread = unread;
    status->slots_free = free_slots;
    status->arena_free_bytes = (int64_t)server->heap.free_bytes;
    status->arena_bytes = (int64_t)server->heap.total;
    status->rounds = (int64_t)server->last_ctl.stats[0];
    status->evals = (int64_t)server->last_ctl.stats[1];
    status->accepts = (int64_t)server->last_ctl.stats[2];
    status->finished = (int64_t)server->finished_total;
    status->busy_ms = server->busy_ms;
    status->launches = server->launches;
    status->smem_bytes = (int32_t)server->smem;
    return HEA_OK;
}

void hea_server_destroy(hea_server *server) { delete server; }

}  // extern "C"
