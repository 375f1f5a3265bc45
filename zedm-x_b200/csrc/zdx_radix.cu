// zdx_radix.cu -- see zdx_radix.cuh.
#include "zdx_radix.cuh"

namespace zdx {

namespace {
constexpr int RT = 256;               // threads per block
constexpr int RI = 8;                 // chunks of RT elements per tile
constexpr int TILE = RT * RI;
constexpr unsigned FULLM = 0xffffffffu;

__global__ void k_rs_hist(const uint32_t* keys, int64_t n, int shift, int nb, int* hist) {
    __shared__ int h[256];
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

__global__ void k_rs_scan(int* hist, int64_t total) {
    __shared__ int ws[32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int64_t base = 0; base < total; base += blockDim.x) {
        int64_t i = base + threadIdx.x;
        int v = i < total ? hist[i] : 0;
        int x = v;
        for (int d = 1; d < 32; d <<= 1) {
            int y = __shfl_up_sync(FULLM, x, d);
            if (lane >= d) x += y;
        }
        if (lane == 31) ws[w] = x;
        __syncthreads();
        if (w == 0) {
            int s = lane < (int)(blockDim.x >> 5) ? ws[lane] : 0;
            for (int d = 1; d < 32; d <<= 1) {
                int y = __shfl_up_sync(FULLM, s, d);
                if (lane >= d) s += y;
            }
            ws[lane] = s;
        }
        __syncthreads();
        int incl = x + (w > 0 ? ws[w - 1] : 0) + carry;
        if (i < total) hist[i] = incl - v;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = incl;
        __syncthreads();
    }
}

__global__ void k_rs_scatter(const uint32_t* kin, const int32_t* vin, uint32_t* kout, int32_t* vout, int64_t n,
                             int shift, int nb, const int* hist) {
    __shared__ int base[256];
    __shared__ int run[256];
    __shared__ int wc[RT / 32][256];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    base[threadIdx.x] = hist[threadIdx.x * nb + blockIdx.x];
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
            int64_t pos = (int64_t)base[d] + run[d] + before + wr;
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
}  // namespace

size_t radix_scratch_bytes(int64_t n) {
    int64_t nb = (n + TILE - 1) / TILE;
    return sizeof(int) * 256 * (size_t)(nb > 0 ? nb : 1);
}

cudaError_t radix_sort_u32(uint32_t* keys, int32_t* vals, uint32_t* kt, int32_t* vt, int64_t n, int key_bits,
                           void* scratch, cudaStream_t s) {
    if (n <= 1) return cudaSuccess;
    const int nb = (int)((n + TILE - 1) / TILE);
    int* hist = static_cast<int*>(scratch);
    uint32_t* ka = keys;
    int32_t* va = vals;
    uint32_t* kb = kt;
    int32_t* vb = vt;
    int passes = (key_bits + 7) / 8;
    if (passes < 1) passes = 1;
    for (int p = 0; p < passes; ++p) {
        int shift = 8 * p;
        k_rs_hist<<<nb, RT, 0, s>>>(ka, n, shift, nb, hist);
        k_rs_scan<<<1, 1024, 0, s>>>(hist, (int64_t)256 * nb);
        k_rs_scatter<<<nb, RT, 0, s>>>(ka, va, kb, vb, n, shift, nb, hist);
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
