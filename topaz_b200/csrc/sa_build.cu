// sa_build.cu -- the suffix array of a .psq text on the device, for
// `topaz index` (serif_index / create_index, src/index.c:24-93, which builds
// it on the host with SA-IS).
//
// Prefix doubling: sort the suffixes by their first 8 bytes, then, while
// two suffixes share a rank, by (rank of i, rank of i + h) for h = 8, 16,
// 32, ...  Ranks are dense (1..n, 0 past the end of the text), so the order
// is the byte-lexicographic suffix order with a shorter suffix first on a
// common prefix -- the order of the reference's SA.  Each round is one
// radix sort of (key, suffix) pairs over only the bits the ranks need, a
// head-flag pass, a scan and a scatter of the new ranks.
#include <algorithm>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "tpz_common.cuh"

namespace {

__global__ void prefix_key_kernel(const uint8_t *T, int64_t n, uint64_t *key, uint32_t *idx) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        // the first 8 bytes, big-endian; bytes past the end are 0, below
        // every .psq byte ('\n' and the letters are nonzero)
        uint64_t k = 0;
#pragma unroll
        for (int b = 0; b < 8; ++b) k = (k << 8) | (i + b < n ? T[i + b] : 0u);
        key[i] = k;
        idx[i] = (uint32_t)i;
    }
}

__global__ void head_kernel(const uint64_t *key, int64_t n, uint32_t *flag) {
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n;
         j += (int64_t)gridDim.x * blockDim.x)
        flag[j] = (j == 0 || key[j] != key[j - 1]) ? 1u : 0u;
}

__global__ void scatter_rank_kernel(const uint32_t *sa, const uint32_t *dense, int64_t n,
                                    uint32_t *rank) {
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n;
         j += (int64_t)gridDim.x * blockDim.x)
        rank[sa[j]] = dense[j];
}

__global__ void pair_key_kernel(const uint32_t *rank, int64_t n, int64_t h, int rbits,
                                uint64_t *key, uint32_t *idx) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        key[i] = ((uint64_t)rank[i] << rbits) | (i + h < n ? rank[i + h] : 0u);
        idx[i] = (uint32_t)i;
    }
}

__global__ void widen_kernel(const uint32_t *sa, int64_t n, int64_t *out) {
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n;
         j += (int64_t)gridDim.x * blockDim.x)
        out[j] = sa[j];
}

struct Bufs {
    std::vector<void *> p;
    ~Bufs() { for (void *q : p) cudaFree(q); }
    template <class T>
    int alloc(T **q, size_t count) {
        void *v = nullptr;
        TPZ_CUDA(cudaMalloc(&v, std::max<size_t>(count * sizeof(T), 16)));
        p.push_back(v);
        *q = (T *)v;
        return TPZ_OK;
    }
};

}  // namespace

extern "C" int tpz_sa_build(const uint8_t *T, int64_t n, int64_t *SA, int32_t *rounds) {
    if (n < 0 || (n > 0 && (!T || !SA))) {
        tpz::set_error("tpz_sa_build: bad arguments");
        return TPZ_E_ARG;
    }
    if (rounds) *rounds = 0;
    if (n == 0) return TPZ_OK;
    if (n >= (int64_t)UINT32_MAX) {
        tpz::set_error("tpz_sa_build: texts of 2^32 - 1 bytes or more are not supported");
        return TPZ_E_RANGE;
    }
    cudaStream_t st = cudaStreamPerThread;
    Bufs b;
    uint8_t *dT; uint64_t *k0, *k1; uint32_t *v0, *v1, *rank, *flag, *dense; void *tmp = nullptr;
    int rc;
    if ((rc = b.alloc(&dT, n)) || (rc = b.alloc(&k0, n)) || (rc = b.alloc(&k1, n)) ||
        (rc = b.alloc(&v0, n)) || (rc = b.alloc(&v1, n)) || (rc = b.alloc(&rank, n)) ||
        (rc = b.alloc(&flag, n)) || (rc = b.alloc(&dense, n)))
        return rc;
    size_t tsort = 0, tscan = 0;
    {
        cub::DoubleBuffer<uint64_t> kk(k0, k1);
        cub::DoubleBuffer<uint32_t> vv(v0, v1);
        TPZ_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tsort, kk, vv, n, 0, 64, st));
        TPZ_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tscan, flag, dense, n, st));
    }
    size_t tbytes = std::max(tsort, tscan);
    if ((rc = b.alloc((uint8_t **)&tmp, tbytes))) return rc;
    TPZ_CUDA(cudaMemcpyAsync(dT, T, n, cudaMemcpyHostToDevice, st));
    const int grid = (int)std::min<int64_t>((n + 255) / 256, (int64_t)tpz::sm_count() * 32);

    int rbits = 1;
    while (((int64_t)1 << rbits) <= n) ++rbits;   // ranks are 0..n
    prefix_key_kernel<<<grid, 256, 0, st>>>(dT, n, k0, v0);
    int begin = 0, end = 64;
    uint64_t *kin = k0, *kalt = k1;
    uint32_t *vin = v0, *valt = v1;
    int nr = 0;
    for (int64_t h = 8;; h *= 2) {
        cub::DoubleBuffer<uint64_t> kk(kin, kalt);
        cub::DoubleBuffer<uint32_t> vv(vin, valt);
        size_t t = tbytes;
        TPZ_CUDA(cub::DeviceRadixSort::SortPairs(tmp, t, kk, vv, n, begin, end, st));
        ++nr;
        head_kernel<<<grid, 256, 0, st>>>(kk.Current(), n, flag);
        t = tbytes;
        TPZ_CUDA(cub::DeviceScan::InclusiveSum(tmp, t, flag, dense, n, st));
        uint32_t distinct = 0;
        TPZ_CUDA(cudaMemcpyAsync(&distinct, dense + n - 1, 4, cudaMemcpyDeviceToHost, st));
        TPZ_CUDA(cudaStreamSynchronize(st));
        if ((int64_t)distinct == n || h >= n) {
            // every suffix has its own rank: the sorted suffixes are the SA
            int64_t *out = reinterpret_cast<int64_t *>(kk.Alternate());
            widen_kernel<<<grid, 256, 0, st>>>(vv.Current(), n, out);
            TPZ_CUDA(cudaMemcpyAsync(SA, out, sizeof(int64_t) * n, cudaMemcpyDeviceToHost, st));
            TPZ_CUDA(cudaStreamSynchronize(st));
            break;
        }
        scatter_rank_kernel<<<grid, 256, 0, st>>>(vv.Current(), dense, n, rank);
        kin = kk.Alternate(); kalt = kk.Current();
        vin = vv.Alternate(); valt = vv.Current();
        pair_key_kernel<<<grid, 256, 0, st>>>(rank, n, h, rbits, kin, vin);
        begin = 0;
        end = 2 * rbits;
    }
    TPZ_CUDA(cudaGetLastError());
    if (rounds) *rounds = nr;
    return TPZ_OK;
}
