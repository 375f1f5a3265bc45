// zdx_radix.cu -- see zdx_radix.cuh.
#include "zdx_radix.cuh"

#include <algorithm>

namespace zdx {

namespace {
constexpr int RT = 256;               // threads per block
constexpr int RI = 8;                 // chunks of RT elements per tile
constexpr int TILE = RT * RI;
constexpr unsigned FULLM = 0xffffffffu;

__device__ __forceinline__ int64_t count_of(int64_t n, const int64_t* n_dev) {
    if (!n_dev) return n;
    const int64_t d = *n_dev;
    return d < n ? d : n;
}

__global__ void k_rs_hist(const uint32_t* keys, int64_t n, const int64_t* n_dev, int shift, int nb, int* hist) {
    __shared__ int h[256];
    n = count_of(n, n_dev);
    h[threadIdx.x] = 0;
    __syncthreads();
    int64_t base = (int64_t)blockIdx.x * TILE;
    for (int k = 0; k < RI; ++k) {
        int64_t i = base + (int64_t)k * RT + threadIdx.x;
        if (i < n) atomicAdd(&h[(keys[i] >> shift) & 255u], 1);
    }
    __syncthreads();
    hist[threadIdx.x * nb + blockIdx.x] = h[threadIdx.x];
}

__global__ void k_rs_scatter(const uint32_t* kin, const int32_t* vin, uint32_t* kout, int32_t* vout, int64_t n,
                             const int64_t* n_dev, int shift, int nb, const int64_t* hoff) {
    __shared__ int64_t base[256];
    n = count_of(n, n_dev);
    __shared__ int run[256];
    __shared__ int wc[RT / 32][256];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    base[threadIdx.x] = hoff[threadIdx.x * nb + blockIdx.x];
    run[threadIdx.x] = 0;
    const int64_t tile = (int64_t)blockIdx.x * TILE;
    for (int k = 0; k < RI; ++k) {
        for (int q = threadIdx.x; q < (RT / 32) * 256; q += RT) wc[q / 256][q % 256] = 0;
        __syncthreads();
        int64_t i = tile + (int64_t)k * RT + threadIdx.x;
        bool ok = i < n;
        uint32_t key = ok ? kin[i] : 0u;
        int d = ok ? (int)((key >> shift) & 255u) : 256;
        unsigned peers = __match_any_sync(FULLM, d);
        int wr = __popc(peers & ((1u << lane) - 1u));
        if (ok && wr == 0) wc[w][d] = __popc(peers);
        __syncthreads();
        if (ok) {
            int before = 0;
            for (int q = 0; q < w; ++q) before += wc[q][d];
            int64_t pos = base[d] + run[d] + before + wr;
            kout[pos] = key;
            vout[pos] = vin[i];
        }
        __syncthreads();
        {
            int t = 0;
            for (int q = 0; q < RT / 32; ++q) t += wc[q][threadIdx.x];
            run[threadIdx.x] += t;
        }
        __syncthreads();
    }
}

template <class T>
__global__ void k_scan_small(const T* cnt, int64_t n, int64_t* off) {
    __shared__ int64_t ws[32];
    __shared__ int64_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int64_t b = 0; b < n; b += blockDim.x) {
        int64_t i = b + threadIdx.x;
        int64_t v = i < n ? (int64_t)cnt[i] : 0;
        int64_t x = v;
        for (int d = 1; d < 32; d <<= 1) {
            int64_t y = __shfl_up_sync(FULLM, x, d);
            if (lane >= d) x += y;
        }
        if (lane == 31) ws[w] = x;
        __syncthreads();
        if (w == 0) {
            int64_t s = lane < (int)(blockDim.x >> 5) ? ws[lane] : 0;
            for (int d = 1; d < 32; d <<= 1) {
                int64_t y = __shfl_up_sync(FULLM, s, d);
                if (lane >= d) s += y;
            }
            ws[lane] = s;
        }
        __syncthreads();
        int64_t incl = x + (w > 0 ? ws[w - 1] : 0) + carry;
        if (i < n) off[i] = incl - v;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) off[n] = carry;
}
// Multi-block exclusive scan of counts into offsets: per-tile sums, one scan of the tile sums, then
// each tile scans itself from its base.  Counts beyond the (device) element count read as zero.
constexpr int ST = 256;            // threads
constexpr int SI = 16;             // elements per thread
constexpr int STILE = ST * SI;

template <class T>
__device__ __forceinline__ int64_t block_excl_scan(int64_t v, int64_t* ws, int64_t& total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int64_t x = v;
    for (int d = 1; d < 32; d <<= 1) {
        int64_t y = __shfl_up_sync(FULLM, x, d);
        if (lane >= d) x += y;
    }
    if (lane == 31) ws[w] = x;
    __syncthreads();
    if (w == 0) {
        int64_t s2 = lane < (ST >> 5) ? ws[lane] : 0;
        for (int d = 1; d < 32; d <<= 1) {
            int64_t y = __shfl_up_sync(FULLM, s2, d);
            if (lane >= d) s2 += y;
        }
        ws[lane] = s2;
    }
    __syncthreads();
    const int64_t incl = x + (w > 0 ? ws[w - 1] : 0);
    total = ws[(ST >> 5) - 1];
    __syncthreads();
    return incl - v;
}

template <class T>
__global__ void __launch_bounds__(ST) k_scan_tiles(const T* cnt, int64_t ncap, const int64_t* n_dev, int64_t* tile_sum) {
    __shared__ int64_t ws[32];
    const int64_t n = count_of(ncap, n_dev);
    const int64_t base = (int64_t)blockIdx.x * STILE + (int64_t)threadIdx.x * SI;
    int64_t v = 0;
    for (int k = 0; k < SI; ++k)
        if (base + k < n) v += (int64_t)cnt[base + k];
    int64_t total;
    block_excl_scan<T>(v, ws, total);
    if (threadIdx.x == 0) tile_sum[blockIdx.x] = total;
}

__global__ void __launch_bounds__(1024) k_scan_tile_sums(int64_t* tile_sum, int nb, const int64_t* n_dev, int64_t ncap,
                                                         int64_t* off) {
    __shared__ int64_t ws[32];
    __shared__ int64_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int b = 0; b < nb; b += blockDim.x) {
        const int i = b + threadIdx.x;
        const int64_t v = i < nb ? tile_sum[i] : 0;
        int64_t x = v;
        for (int d = 1; d < 32; d <<= 1) {
            int64_t y = __shfl_up_sync(FULLM, x, d);
            if (lane >= d) x += y;
        }
        if (lane == 31) ws[w] = x;
        __syncthreads();
        if (w == 0) {
            int64_t s2 = lane < (int)(blockDim.x >> 5) ? ws[lane] : 0;
            for (int d = 1; d < 32; d <<= 1) {
                int64_t y = __shfl_up_sync(FULLM, s2, d);
                if (lane >= d) s2 += y;
            }
            ws[lane] = s2;
        }
        __syncthreads();
        const int64_t incl = x + (w > 0 ? ws[w - 1] : 0) + carry;
        if (i < nb) tile_sum[i] = incl - v;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) off[count_of(ncap, n_dev)] = carry;
}

template <class T>
__global__ void __launch_bounds__(ST) k_scan_apply(const T* cnt, int64_t ncap, const int64_t* n_dev,
                                                   const int64_t* tile_base, int64_t* off) {
    __shared__ int64_t ws[32];
    const int64_t n = count_of(ncap, n_dev);
    const int64_t base = (int64_t)blockIdx.x * STILE + (int64_t)threadIdx.x * SI;
    if ((int64_t)blockIdx.x * STILE >= n) return;  // whole block beyond n: uniform exit
    T c[SI];
    int64_t v = 0;
    for (int k = 0; k < SI; ++k) {
        c[k] = base + k < n ? cnt[base + k] : T(0);
        v += (int64_t)c[k];
    }
    int64_t total;
    int64_t run = block_excl_scan<T>(v, ws, total) + tile_base[blockIdx.x];
    for (int k = 0; k < SI; ++k) {
        if (base + k < n) off[base + k] = run;
        run += (int64_t)c[k];
    }
}

// the whole scan in one block when it fits one tile (small scenes: one launch instead of three)
template <class T>
__global__ void __launch_bounds__(ST) k_scan_one(const T* cnt, int64_t ncap, const int64_t* n_dev, int64_t* off) {
    __shared__ int64_t ws[32];
    const int64_t n = count_of(ncap, n_dev);
    const int64_t base = (int64_t)threadIdx.x * SI;
    T c[SI];
    int64_t v = 0;
    for (int k = 0; k < SI; ++k) {
        c[k] = base + k < n ? cnt[base + k] : T(0);
        v += (int64_t)c[k];
    }
    int64_t total;
    int64_t run = block_excl_scan<T>(v, ws, total);
    for (int k = 0; k < SI; ++k) {
        if (base + k < n) off[base + k] = run;
        run += (int64_t)c[k];
    }
    if (threadIdx.x == 0) off[n] = total;
}
}  // namespace

int scan_kernels(int64_t ncap) { return ncap <= STILE ? 1 : 3; }

int radix_kernels(int64_t n, int key_bits) {
    if (n <= 0) return 0;
    const int64_t nb = (n + TILE - 1) / TILE;
    const int passes = std::max(1, (key_bits + 7) / 8);
    return passes * (2 + scan_kernels(256 * nb));
}

size_t scan_scratch_bytes(int64_t ncap) {
    const int64_t nb = (ncap + STILE - 1) / STILE;
    return sizeof(int64_t) * (size_t)(nb > 0 ? nb : 1);
}

template <class T>
cudaError_t scan_offsets(const T* cnt, int64_t ncap, const int64_t* n_dev, int64_t* off, void* scratch, cudaStream_t s) {
    const int nb = (int)std::max<int64_t>(1, (ncap + STILE - 1) / STILE);
    if (nb == 1) {
        k_scan_one<T><<<1, ST, 0, s>>>(cnt, ncap, n_dev, off);
        return cudaGetLastError();
    }
    int64_t* ts = static_cast<int64_t*>(scratch);
    k_scan_tiles<T><<<nb, ST, 0, s>>>(cnt, ncap, n_dev, ts);
    k_scan_tile_sums<<<1, 1024, 0, s>>>(ts, nb, n_dev, ncap, off);
    k_scan_apply<T><<<nb, ST, 0, s>>>(cnt, ncap, n_dev, ts, off);
    return cudaGetLastError();
}
template cudaError_t scan_offsets<int32_t>(const int32_t*, int64_t, const int64_t*, int64_t*, void*, cudaStream_t);
template cudaError_t scan_offsets<int64_t>(const int64_t*, int64_t, const int64_t*, int64_t*, void*, cudaStream_t);

// scratch: digit histogram (int, 256 x tiles), its offsets (int64, 256 x tiles + 1), the scan's tile sums
static size_t radix_parts(int64_t n, size_t* off_at, size_t* tmp_at) {
    const int64_t nb = std::max<int64_t>(1, (n + TILE - 1) / TILE);
    const size_t h = (sizeof(int) * 256 * (size_t)nb + 15) & ~size_t(15);
    const size_t o = (sizeof(int64_t) * (256 * (size_t)nb + 1) + 15) & ~size_t(15);
    if (off_at) *off_at = h;
    if (tmp_at) *tmp_at = h + o;
    return h + o + scan_scratch_bytes(256 * nb);
}
size_t radix_scratch_bytes(int64_t n) { return radix_parts(n, nullptr, nullptr); }

cudaError_t radix_sort_u32(uint32_t* keys, int32_t* vals, uint32_t* kt, int32_t* vt, int64_t n, int key_bits,
                           void* scratch, cudaStream_t s, const int64_t* n_dev) {
    if (n <= 1 && !n_dev) return cudaSuccess;
    if (n <= 0) return cudaSuccess;
    const int nb = (int)((n + TILE - 1) / TILE);
    size_t off_at = 0, tmp_at = 0;
    radix_parts(n, &off_at, &tmp_at);
    int* hist = static_cast<int*>(scratch);
    int64_t* hoff = reinterpret_cast<int64_t*>(static_cast<char*>(scratch) + off_at);
    void* stmp = static_cast<char*>(scratch) + tmp_at;
    uint32_t* ka = keys;
    int32_t* va = vals;
    uint32_t* kb = kt;
    int32_t* vb = vt;
    int passes = (key_bits + 7) / 8;
    if (passes < 1) passes = 1;
    for (int p = 0; p < passes; ++p) {
        int shift = 8 * p;
        k_rs_hist<<<nb, RT, 0, s>>>(ka, n, n_dev, shift, nb, hist);
        scan_offsets<int32_t>(hist, (int64_t)256 * nb, nullptr, hoff, stmp, s);
        k_rs_scatter<<<nb, RT, 0, s>>>(ka, va, kb, vb, n, n_dev, shift, nb, hoff);
        uint32_t* tk = ka;
        ka = kb;
        kb = tk;
        int32_t* tv = va;
        va = vb;
        vb = tv;
    }
    if (ka != keys) {
        cudaMemcpyAsync(keys, ka, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(vals, va, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, s);
    }
    return cudaGetLastError();
}

cudaError_t scan_counts_i32(const int32_t* cnt, int64_t n, int64_t* off, cudaStream_t s) {
    k_scan_small<int32_t><<<1, 1024, 0, s>>>(cnt, n, off);
    return cudaGetLastError();
}

}  // namespace zdx
