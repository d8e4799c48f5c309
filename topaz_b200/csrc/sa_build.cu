// sa_build.cu -- the suffix array of a .psq text on the device, for
// `topaz index` (serif_index / create_index, src/index.c:24-93, build it on
// the host with divsufsort64).  The order is byte-lexicographic with a
// shorter suffix first on a common prefix -- the reference's .SA (a text's
// suffix array is unique, so any exact construction writes the same bytes).
//
// Built for texts of any size up to what HBM holds (64-bit positions,
// ~10 G residues on one B200), in two phases:
//
// Partitions.  Every suffix gets a key of its first c symbols (bytes ranked
// among the values present, 0 past the end of the text), packed b bits each
// into a 64-bit word (27 symbols for a .psq: b = 5, c = 12).  The suffixes
// are split by their first q symbols into partitions that fit the free
// device memory; partitions are contiguous row ranges of the final array.
// Per partition: a selection pass over the text, one radix sort of
// (key, position) pairs, then rounds that re-sort only the runs of equal keys
// by their next c symbols (segmented sorts), for a bounded number of rounds.
// The sorted rows go to the caller's sink as they are done.  Random text
// leaves no runs after two or three rounds.
//
// Doubling.  Runs still tied after the partition rounds (long repeats) are
// finished by prefix doubling (Larsson-Sadakane): the inverse array ISA holds
// for every suffix its final row, or the first row of its tied run, so two
// suffixes tied on their first h symbols are ordered by ISA at +h, and each
// round doubles h.  Their final rows go to the sink last.
#include <string.h>

#include <algorithm>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_segmented_sort.cuh>
#include <cub/device/device_select.cuh>
#include <thrust/iterator/counting_iterator.h>

#include "tpz_common.cuh"

namespace {

constexpr int kRefineRounds = 8;          // key-extension rounds per partition
constexpr int kHistMaxBins = 32768;       // partition codes (first q symbols)

struct SymTab {
    uint8_t sym[256];    // byte -> symbol 1..K-1 (0 = past the end of the text)
    int bits;            // bits per symbol
    int per_key;         // symbols per 64-bit key
    int q;               // symbols of the partition code
    int K;               // symbol count including the end symbol
};

__device__ __forceinline__ uint32_t sym_at(const uint8_t *T, int64_t n, int64_t p, const SymTab &s) {
    return p < n ? s.sym[T[p]] : 0u;
}

__device__ __forceinline__ uint64_t key_at(const uint8_t *T, int64_t n, int64_t i, const SymTab &s) {
    uint64_t k = 0;
    for (int t = 0; t < s.per_key; ++t) k = (k << s.bits) | sym_at(T, n, i + t, s);
    return k;
}

__device__ __forceinline__ uint32_t code_at(const uint8_t *T, int64_t n, int64_t i, const SymTab &s) {
    uint32_t c = 0;
    for (int t = 0; t < s.q; ++t) c = c * s.K + sym_at(T, n, i + t, s);
    return c;
}

__global__ void byte_hist_kernel(const uint8_t *T, int64_t n, unsigned long long *cnt) {
    __shared__ unsigned int h[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) h[i] = 0;
    __syncthreads();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        atomicAdd(&h[T[i]], 1u);
    __syncthreads();
    for (int i = threadIdx.x; i < 256; i += blockDim.x)
        if (h[i]) atomicAdd(&cnt[i], (unsigned long long)h[i]);
}

// suffixes per partition code; per-block counts in shared memory
__global__ void code_hist_kernel(const uint8_t *T, int64_t n, const __grid_constant__ SymTab s,
                                 int nbins, unsigned long long *cnt) {
    extern __shared__ unsigned int hs[];
    for (int i = threadIdx.x; i < nbins; i += blockDim.x) hs[i] = 0;
    __syncthreads();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        atomicAdd(&hs[code_at(T, n, i, s)], 1u);
    __syncthreads();
    for (int i = threadIdx.x; i < nbins; i += blockDim.x)
        if (hs[i]) atomicAdd(&cnt[i], (unsigned long long)hs[i]);
}

// (key, position) of every suffix whose code lies in [lo, hi), in any order
__global__ void select_kernel(const uint8_t *T, int64_t n, const __grid_constant__ SymTab s,
                              uint32_t lo, uint32_t hi, uint64_t *key, int64_t *pos,
                              unsigned long long *count) {
    const int lane = threadIdx.x & 31;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    // whole warps step through the text together so the ballot sees 32 lanes
    for (int64_t base = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) - lane; base < n;
         base += stride) {
        const int64_t i = base + lane;
        bool take = false;
        if (i < n) {
            const uint32_t c = code_at(T, n, i, s);
            take = c >= lo && c < hi;
        }
        const unsigned m = __ballot_sync(0xFFFFFFFFu, take);
        if (!m) continue;
        unsigned long long slot = 0;
        if (lane == 0) slot = atomicAdd(count, (unsigned long long)__popc(m));
        slot = __shfl_sync(0xFFFFFFFFu, slot, 0);
        if (take) {
            const unsigned long long k = slot + __popc(m & ((1u << lane) - 1u));
            key[k] = key_at(T, n, i, s);
            pos[k] = i;
        }
    }
}

// flags of the sorted partition: tie[k] = key equal to a neighbour's;
// head[k] = first of a run of equal keys (only set on tied entries)
__global__ void tie_flags_kernel(const uint64_t *key, int64_t m, uint8_t *tie, uint8_t *head) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < m;
         k += (int64_t)gridDim.x * blockDim.x) {
        const bool prev = k > 0 && key[k] == key[k - 1];
        const bool next = k + 1 < m && key[k] == key[k + 1];
        tie[k] = prev || next;
        head[k] = (!prev && next) ? 1 : 0;
    }
}

// the same over a compacted run list: entries x, x+1 are tied when they sit
// in the same run and carry equal keys
__global__ void tie_flags_runs_kernel(const uint64_t *key, const int32_t *run, int64_t u,
                                      uint8_t *tie, uint8_t *head) {
    for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < u;
         x += (int64_t)gridDim.x * blockDim.x) {
        const bool prev = x > 0 && run[x] == run[x - 1] && key[x] == key[x - 1];
        const bool next = x + 1 < u && run[x] == run[x + 1] && key[x] == key[x + 1];
        tie[x] = prev || next;
        head[x] = (!prev && next) ? 1 : 0;
    }
}

__global__ void iota64_kernel(int64_t *v, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        v[i] = i;
}

__global__ void widen_flags_kernel(const uint8_t *f, int64_t u, int32_t *w) {
    for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < u;
         x += (int64_t)gridDim.x * blockDim.x)
        w[x] = f[x];
}

__global__ void minus_one_kernel(int32_t *v, int64_t u) {
    for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < u;
         x += (int64_t)gridDim.x * blockDim.x)
        v[x] -= 1;
}

// run start offsets: off[r] = first entry of run r (from the head indices)
__global__ void run_off_kernel(const int64_t *head_x, int32_t nruns, int64_t u, int32_t *off) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r <= nruns;
         r += (int64_t)gridDim.x * blockDim.x)
        off[r] = r < nruns ? (int32_t)head_x[r] : (int32_t)u;
}

// In-place compaction of the tied list to the entries sel[0..u2) (sel
// increasing, so each entry moves down or stays): one block walks the list
// in chunks, reading a chunk completely before writing it.
__global__ void compact_kernel(const int64_t *sel, int64_t u2, int64_t *ukpos, int64_t *upos,
                               const int64_t *upos_sorted, uint8_t *uhead, const uint8_t *uhead_new) {
    for (int64_t c = 0; c < u2; c += blockDim.x) {
        const int64_t x = c + threadIdx.x;
        int64_t kp = 0, p = 0;
        uint8_t h = 0;
        if (x < u2) {
            const int64_t y = sel[x];
            kp = ukpos[y];
            p = upos_sorted[y];
            h = uhead_new[y];
        }
        __syncthreads();
        if (x < u2) { ukpos[x] = kp; upos[x] = p; uhead[x] = h; }
        __syncthreads();
    }
}

__global__ void dbl_compact_kernel(const int64_t *sel, int64_t u2, int64_t *brow, int64_t *bidx,
                                   const int64_t *ng, int64_t *bslot, int64_t *bgrp) {
    for (int64_t c = 0; c < u2; c += blockDim.x) {
        const int64_t x = c + threadIdx.x;
        int64_t r = 0, i = 0, g = 0, sl = 0;
        if (x < u2) {
            const int64_t y = sel[x];
            r = brow[y]; i = bidx[y]; g = ng[y]; sl = bslot[y];
        }
        __syncthreads();
        if (x < u2) { brow[x] = r; bidx[x] = i; bgrp[x] = g; bslot[x] = sl; }
        __syncthreads();
    }
}

// next key of each tied entry: its suffix's symbols at depth d
__global__ void next_key_kernel(const uint8_t *T, int64_t n, const __grid_constant__ SymTab s,
                                const int64_t *pos, int64_t u, int64_t d, uint64_t *key) {
    for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < u;
         x += (int64_t)gridDim.x * blockDim.x)
        key[x] = key_at(T, n, pos[x] + d, s);
}

template <class T>
__global__ void gather_kernel(const T *src, const int64_t *at, int64_t u, T *dst) {
    for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < u;
         x += (int64_t)gridDim.x * blockDim.x)
        dst[x] = src[at[x]];
}

template <class T>
__global__ void scatter_kernel(const T *src, const int64_t *at, int64_t u, T *dst) {
    for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < u;
         x += (int64_t)gridDim.x * blockDim.x)
        dst[at[x]] = src[x];
}

// ISA of a finished partition: every suffix at its row
__global__ void isa_rows_kernel(const int64_t *pos, int64_t m, int64_t base, int64_t *isa) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < m;
         k += (int64_t)gridDim.x * blockDim.x)
        isa[pos[k]] = base + k;
}

// entries still tied after the partition rounds: row, suffix, first row of
// the tied run (the run's ISA value) -- appended to the doubling list
__global__ void tied_out_kernel(const int64_t *ukpos, const int64_t *upos, const int32_t *run,
                                const int32_t *off, int64_t u, int64_t base, int64_t *isa,
                                int64_t *brow, int64_t *bidx, int64_t *bgrp) {
    for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < u;
         x += (int64_t)gridDim.x * blockDim.x) {
        const int64_t g = base + ukpos[off[run[x]]];
        brow[x] = base + ukpos[x];
        bidx[x] = upos[x];
        bgrp[x] = g;
        isa[upos[x]] = g;
    }
}

// doubling: the key of a tied suffix is the ISA value h positions on
// (+1; 0 past the end of the text, which sorts first)
__global__ void dbl_key_kernel(const int64_t *bidx, int64_t u, int64_t h, int64_t n,
                               const int64_t *isa, uint64_t *key) {
    for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < u;
         x += (int64_t)gridDim.x * blockDim.x) {
        const int64_t j = bidx[x] + h;
        key[x] = j < n ? (uint64_t)isa[j] + 1 : 0;
    }
}

// segment starts of the doubling list (runs = equal bgrp, contiguous)
__global__ void dbl_heads_kernel(const int64_t *bgrp, int64_t u, uint8_t *head) {
    for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < u;
         x += (int64_t)gridDim.x * blockDim.x)
        head[x] = (x == 0 || bgrp[x] != bgrp[x - 1]) ? 1 : 0;
}

// after the sort: the new run of x starts at the first entry of its old run
// with the same key; rows of a run are consecutive, so that entry's row is
// the largest "starts a new run here" row at or before x
__global__ void dbl_mark_kernel(const int64_t *bgrp, const uint64_t *key, const int64_t *brow,
                                int64_t u, int64_t *mark) {
    for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < u;
         x += (int64_t)gridDim.x * blockDim.x) {
        const bool start = x == 0 || bgrp[x] != bgrp[x - 1] || key[x] != key[x - 1];
        mark[x] = start ? brow[x] : -1;
    }
}

struct MaxOp {
    __device__ __forceinline__ int64_t operator()(int64_t a, int64_t b) const { return a > b ? a : b; }
};

__global__ void dbl_update_kernel(const int64_t *ng, const int64_t *bidx, const int64_t *brow,
                                  const int64_t *bslot, int64_t u, int64_t *isa, int64_t *fix,
                                  uint8_t *keep) {
    for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < u;
         x += (int64_t)gridDim.x * blockDim.x) {
        const bool tied = (x > 0 && ng[x] == ng[x - 1]) || (x + 1 < u && ng[x] == ng[x + 1]);
        isa[bidx[x]] = tied ? ng[x] : brow[x];
        fix[bslot[x]] = bidx[x];
        keep[x] = tied;
    }
}

// stream-ordered device allocations, freed together
struct Mem {
    std::vector<void *> p;
    cudaStream_t st;
    explicit Mem(cudaStream_t s) : st(s) {}
    ~Mem() { for (void *q : p) cudaFreeAsync(q, st); }
    template <class T>
    int alloc(T **q, size_t count) {
        void *v = nullptr;
        TPZ_CUDA(cudaMallocAsync(&v, std::max<size_t>(count * sizeof(T), 16), st));
        p.push_back(v);
        *q = (T *)v;
        return TPZ_OK;
    }
};

int grid_for(int64_t n) {
    return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)tpz::sm_count() * 16));
}

// Copies device rows to the sink through a pinned staging buffer.
struct Emitter {
    tpz_sa_sink sink;
    void *user;
    int64_t *stage = nullptr;
    int64_t cap = 0;
    ~Emitter() { if (stage) cudaFreeHost(stage); }
    int init(int64_t c) {
        cap = c;
        TPZ_CUDA(cudaMallocHost((void **)&stage, sizeof(int64_t) * cap));
        return TPZ_OK;
    }
    int emit(const int64_t *d, int64_t first_row, int64_t m, cudaStream_t st) {
        for (int64_t a = 0; a < m; a += cap) {
            const int64_t k = std::min(cap, m - a);
            TPZ_CUDA(cudaMemcpyAsync(stage, d + a, sizeof(int64_t) * k, cudaMemcpyDeviceToHost, st));
            TPZ_CUDA(cudaStreamSynchronize(st));
            if (sink(user, first_row + a, stage, k) != 0) {
                tpz::set_error("tpz_sa_build: the sink refused rows");
                return TPZ_E_ARG;
            }
        }
        return TPZ_OK;
    }
};

int host_sink_copy(void *user, int64_t first_row, const int64_t *rows, int64_t count) {
    memcpy((int64_t *)user + first_row, rows, sizeof(int64_t) * count);
    return 0;
}

// Runs of a tied list given its head flags: run[x] = run number of entry x,
// off[0..nruns] = first entry of each run (off[nruns] = u).
int find_runs(Mem &mem, const uint8_t *head, int64_t u, int32_t *run, int32_t *off, int32_t *nruns,
              int32_t *h32, int64_t *hx, int64_t *dn, cudaStream_t st) {
    widen_flags_kernel<<<grid_for(u), 256, 0, st>>>(head, u, h32);
    size_t sb = 0;
    TPZ_CUDA(cub::DeviceScan::InclusiveSum(nullptr, sb, h32, run, u, st));
    uint8_t *stmp;
    int rc;
    if ((rc = mem.alloc(&stmp, sb))) return rc;
    TPZ_CUDA(cub::DeviceScan::InclusiveSum(stmp, sb, h32, run, u, st));
    TPZ_CUDA(cudaMemcpyAsync(nruns, run + u - 1, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    minus_one_kernel<<<grid_for(u), 256, 0, st>>>(run, u);
    thrust::counting_iterator<int64_t> it(0);
    size_t fb = 0;
    TPZ_CUDA(cub::DeviceSelect::Flagged(nullptr, fb, it, head, hx, dn, u, st));
    uint8_t *ftmp;
    if ((rc = mem.alloc(&ftmp, fb))) return rc;
    TPZ_CUDA(cub::DeviceSelect::Flagged(ftmp, fb, it, head, hx, dn, u, st));
    TPZ_CUDA(cudaStreamSynchronize(st));
    run_off_kernel<<<grid_for((int64_t)*nruns + 1), 256, 0, st>>>(hx, *nruns, u, off);
    return TPZ_OK;
}

// Indices x < u with flag[x] set, into sel; their count into *count.
int select_flagged(Mem &mem, const uint8_t *flag, int64_t u, int64_t *sel, int64_t *dn, int64_t *count,
                   cudaStream_t st) {
    thrust::counting_iterator<int64_t> it(0);
    size_t fb = 0;
    TPZ_CUDA(cub::DeviceSelect::Flagged(nullptr, fb, it, flag, sel, dn, u, st));
    uint8_t *ftmp;
    int rc;
    if ((rc = mem.alloc(&ftmp, fb))) return rc;
    TPZ_CUDA(cub::DeviceSelect::Flagged(ftmp, fb, it, flag, sel, dn, u, st));
    TPZ_CUDA(cudaMemcpyAsync(count, dn, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    TPZ_CUDA(cudaStreamSynchronize(st));
    return TPZ_OK;
}

}  // namespace

extern "C" int tpz_sa_build_sink(const uint8_t *T, int64_t n, tpz_sa_sink sink, void *user,
                                 int64_t max_partition, int32_t *rounds) {
    if (n < 0 || (n > 0 && (!T || !sink)) || max_partition < 0) {
        tpz::set_error("tpz_sa_build: bad arguments");
        return TPZ_E_ARG;
    }
    if (rounds) *rounds = 0;
    if (n == 0) return TPZ_OK;
    cudaStream_t st = cudaStreamPerThread;
    Mem mem(st);
    int rc;
    int nr = 0;

    // ---- text and symbol table
    uint8_t *dT;
    unsigned long long *dcnt;
    int64_t *dn;
    if ((rc = mem.alloc(&dT, n)) || (rc = mem.alloc(&dcnt, kHistMaxBins)) || (rc = mem.alloc(&dn, 1)))
        return rc;
    TPZ_CUDA(cudaMemcpyAsync(dT, T, n, cudaMemcpyHostToDevice, st));
    TPZ_CUDA(cudaMemsetAsync(dcnt, 0, sizeof(unsigned long long) * 256, st));
    byte_hist_kernel<<<grid_for(n), 256, 0, st>>>(dT, n, dcnt);
    unsigned long long bh[256];
    TPZ_CUDA(cudaMemcpyAsync(bh, dcnt, sizeof bh, cudaMemcpyDeviceToHost, st));
    TPZ_CUDA(cudaStreamSynchronize(st));
    SymTab s;
    memset(&s, 0, sizeof s);
    int K = 1;
    for (int b = 0; b < 256; ++b)
        if (bh[b]) s.sym[b] = (uint8_t)K++;
    s.K = K;
    s.bits = 1;
    while ((1 << s.bits) < K) ++s.bits;
    s.per_key = 64 / s.bits;
    s.q = 1;
    int nbins = K;
    while (s.q < s.per_key && (int64_t)nbins * K <= kHistMaxBins) { nbins *= K; ++s.q; }
    const int kbits = s.per_key * s.bits;

    // ---- suffixes per partition code
    TPZ_CUDA(cudaMemsetAsync(dcnt, 0, sizeof(unsigned long long) * nbins, st));
    TPZ_CUDA(cudaFuncSetAttribute(code_hist_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  nbins * 4));
    code_hist_kernel<<<grid_for(n), 512, nbins * 4, st>>>(dT, n, s, nbins, dcnt);
    std::vector<unsigned long long> hist(nbins);
    TPZ_CUDA(cudaMemcpyAsync(hist.data(), dcnt, sizeof(unsigned long long) * nbins,
                             cudaMemcpyDeviceToHost, st));
    TPZ_CUDA(cudaStreamSynchronize(st));

    // ---- the inverse array (doubling phase) and the partition capacity:
    // keys and positions double-buffered (32 B per entry) plus the sort's
    // scratch in half of the free memory; the other half is for the lists
    // of tied runs
    int64_t *isa;
    if ((rc = mem.alloc(&isa, n))) return rc;
    TPZ_CUDA(cudaStreamSynchronize(st));
    size_t free_b = 0, total_b = 0;
    TPZ_CUDA(cudaMemGetInfo(&free_b, &total_b));
    int64_t cap = (int64_t)(0.5 * (double)free_b / 32.0);
    if (max_partition > 0) cap = std::min(cap, max_partition);
    cap = std::max<int64_t>(1, std::min(cap, n));
    size_t tmp_bytes = 0;
    for (;;) {
        cub::DoubleBuffer<uint64_t> kk(nullptr, nullptr);
        cub::DoubleBuffer<int64_t> vv(nullptr, nullptr);
        TPZ_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, kk, vv, cap, 0, kbits, st));
        if (32.0 * cap + tmp_bytes <= 0.5 * (double)free_b || cap <= 1024) break;
        cap = cap * 7 / 8;
    }
    int64_t biggest = 0;
    for (unsigned long long h : hist) biggest = std::max<int64_t>(biggest, (int64_t)h);
    if (biggest > cap) {
        tpz::set_error("tpz_sa_build: more suffixes share their first symbols than one device "
                       "sort holds (text too repetitive)");
        return TPZ_E_RANGE;
    }
    uint64_t *k0, *k1;
    int64_t *v0, *v1;
    uint8_t *tmp;
    if ((rc = mem.alloc(&k0, cap)) || (rc = mem.alloc(&k1, cap)) || (rc = mem.alloc(&v0, cap)) ||
        (rc = mem.alloc(&v1, cap)) || (rc = mem.alloc(&tmp, tmp_bytes)))
        return rc;
    Emitter em{sink, user};
    if ((rc = em.init(std::min<int64_t>(n, (int64_t)1 << 25)))) return rc;

    // tied entries left for the doubling phase: row, suffix, run's first row
    std::vector<int64_t *> brow_l, bidx_l, bgrp_l;
    std::vector<int64_t> bn_l;
    int64_t btotal = 0;

    // ---- partitions: consecutive code ranges of at most cap suffixes
    int64_t base = 0;
    for (int lo = 0; lo < nbins;) {
        int hi = lo;
        int64_t m = 0;
        while (hi < nbins && m + (int64_t)hist[hi] <= cap) m += (int64_t)hist[hi++];
        if (m == 0) { lo = hi; continue; }
        Mem pm(st);            // this partition's temporaries
        TPZ_CUDA(cudaMemsetAsync(dcnt, 0, sizeof(unsigned long long), st));
        select_kernel<<<grid_for(n), 256, 0, st>>>(dT, n, s, (uint32_t)lo, (uint32_t)hi, k0, v0, dcnt);
        unsigned long long got = 0;
        TPZ_CUDA(cudaMemcpyAsync(&got, dcnt, sizeof got, cudaMemcpyDeviceToHost, st));
        cub::DoubleBuffer<uint64_t> kk(k0, k1);
        cub::DoubleBuffer<int64_t> vv(v0, v1);
        size_t t = tmp_bytes;
        TPZ_CUDA(cub::DeviceRadixSort::SortPairs(tmp, t, kk, vv, m, 0, kbits, st));
        ++nr;
        TPZ_CUDA(cudaStreamSynchronize(st));
        if ((int64_t)got != m) {
            tpz::set_error("tpz_sa_build: internal error (partition selection)");
            return TPZ_E_DEVICE;
        }
        uint64_t *key = kk.Current();
        int64_t *pos = vv.Current();
        // flags in the other key buffer, the tied entries' partition indices
        // in the other position buffer
        uint8_t *tie = reinterpret_cast<uint8_t *>(kk.Alternate());
        uint8_t *head = tie + m;
        int64_t *ukpos = vv.Alternate();
        tie_flags_kernel<<<grid_for(m), 256, 0, st>>>(key, m, tie, head);
        int64_t u = 0;
        if ((rc = select_flagged(pm, tie, m, ukpos, dn, &u, st))) return rc;
        if (u > INT32_MAX) {
            tpz::set_error("tpz_sa_build: too many tied suffixes in one partition");
            return TPZ_E_RANGE;
        }
        int64_t d = s.per_key;        // symbols every tied entry is known to share
        int64_t *upos = nullptr, *upos2 = nullptr, *hx = nullptr, *sel = nullptr;
        uint64_t *ukey = nullptr, *ukey2 = nullptr;
        int32_t *run = nullptr, *h32 = nullptr, *off = nullptr;
        uint8_t *uhead = nullptr, *utie = nullptr, *uhead2 = nullptr;
        if (u > 0) {
            if ((rc = pm.alloc(&upos, u)) || (rc = pm.alloc(&upos2, u)) || (rc = pm.alloc(&ukey, u)) ||
                (rc = pm.alloc(&ukey2, u)) || (rc = pm.alloc(&run, u)) || (rc = pm.alloc(&h32, u)) ||
                (rc = pm.alloc(&off, u + 1)) || (rc = pm.alloc(&hx, u)) || (rc = pm.alloc(&sel, u)) ||
                (rc = pm.alloc(&uhead, u)) || (rc = pm.alloc(&utie, u)) || (rc = pm.alloc(&uhead2, u))) {
                tpz::set_error("tpz_sa_build: no device memory for the tied runs (text too repetitive)");
                return rc;
            }
            gather_kernel<int64_t><<<grid_for(u), 256, 0, st>>>(pos, ukpos, u, upos);
            gather_kernel<uint8_t><<<grid_for(u), 256, 0, st>>>(head, ukpos, u, uhead);
        }
        for (int round = 0; u > 0 && round < kRefineRounds; ++round) {
            int32_t nruns = 0;
            if ((rc = find_runs(pm, uhead, u, run, off, &nruns, h32, hx, dn, st))) return rc;
            // the next symbols of every tied suffix, sorted within its run
            next_key_kernel<<<grid_for(u), 256, 0, st>>>(dT, n, s, upos, u, d, ukey);
            size_t gb = 0;
            TPZ_CUDA(cub::DeviceSegmentedSort::SortPairs(nullptr, gb, ukey, ukey2, upos, upos2, (int)u,
                                                         nruns, off, off + 1, st));
            uint8_t *gtmp;
            if ((rc = pm.alloc(&gtmp, gb))) return rc;
            TPZ_CUDA(cub::DeviceSegmentedSort::SortPairs(gtmp, gb, ukey, ukey2, upos, upos2, (int)u,
                                                         nruns, off, off + 1, st));
            ++nr;
            d += s.per_key;
            scatter_kernel<int64_t><<<grid_for(u), 256, 0, st>>>(upos2, ukpos, u, pos);
            // still tied: same run and the same next symbols
            tie_flags_runs_kernel<<<grid_for(u), 256, 0, st>>>(ukey2, run, u, utie, uhead2);
            int64_t u2 = 0;
            if ((rc = select_flagged(pm, utie, u, sel, dn, &u2, st))) return rc;
            if (u2 > 0) {
                // compact in place: sel is increasing, so sel[x] >= x
                compact_kernel<<<1, 1024, 0, st>>>(sel, u2, ukpos, upos, upos2, uhead, uhead2);
            }
            u = u2;
        }
        isa_rows_kernel<<<grid_for(m), 256, 0, st>>>(pos, m, base, isa);
        if (u > 0) {
            // runs still tied go to the doubling phase; their ISA is the
            // run's first row
            int32_t nruns = 0;
            if ((rc = find_runs(pm, uhead, u, run, off, &nruns, h32, hx, dn, st))) return rc;
            int64_t *br, *bi, *bg;
            if ((rc = mem.alloc(&br, u)) || (rc = mem.alloc(&bi, u)) || (rc = mem.alloc(&bg, u))) {
                tpz::set_error("tpz_sa_build: no device memory for the tied runs (text too repetitive)");
                return rc;
            }
            tied_out_kernel<<<grid_for(u), 256, 0, st>>>(ukpos, upos, run, off, u, base, isa, br, bi, bg);
            brow_l.push_back(br); bidx_l.push_back(bi); bgrp_l.push_back(bg); bn_l.push_back(u);
            btotal += u;
        }
        TPZ_CUDA(cudaGetLastError());
        // rows of tied runs are written again after the doubling phase
        if ((rc = em.emit(pos, base, m, st))) return rc;
        base += m;
        lo = hi;
    }
    if (base != n) {
        tpz::set_error("tpz_sa_build: internal error (partition sizes)");
        return TPZ_E_DEVICE;
    }

    // ---- doubling phase over the runs still tied
    if (btotal > 0) {
        if (btotal > INT32_MAX) {
            tpz::set_error("tpz_sa_build: too many tied suffixes (text too repetitive)");
            return TPZ_E_RANGE;
        }
        Mem dm(st);
        int64_t u = btotal;
        int64_t *brow, *bidx, *bgrp, *bslot, *fix, *frow, *t64, *mark, *ng, *hx, *sel;
        uint64_t *key, *key2;
        uint8_t *head, *keep;
        int32_t *off;
        if ((rc = dm.alloc(&brow, u)) || (rc = dm.alloc(&bidx, u)) || (rc = dm.alloc(&bgrp, u)) ||
            (rc = dm.alloc(&bslot, u)) || (rc = dm.alloc(&fix, u)) || (rc = dm.alloc(&frow, u)) ||
            (rc = dm.alloc(&t64, u)) || (rc = dm.alloc(&mark, u)) || (rc = dm.alloc(&ng, u)) ||
            (rc = dm.alloc(&hx, u)) || (rc = dm.alloc(&sel, u)) || (rc = dm.alloc(&key, u)) ||
            (rc = dm.alloc(&key2, u)) || (rc = dm.alloc(&head, u)) || (rc = dm.alloc(&keep, u)) ||
            (rc = dm.alloc(&off, u + 1))) {
            tpz::set_error("tpz_sa_build: no device memory for the doubling phase (text too repetitive)");
            return rc;
        }
        int64_t at = 0;
        for (size_t i = 0; i < bn_l.size(); ++i) {
            TPZ_CUDA(cudaMemcpyAsync(brow + at, brow_l[i], 8 * bn_l[i], cudaMemcpyDeviceToDevice, st));
            TPZ_CUDA(cudaMemcpyAsync(bidx + at, bidx_l[i], 8 * bn_l[i], cudaMemcpyDeviceToDevice, st));
            TPZ_CUDA(cudaMemcpyAsync(bgrp + at, bgrp_l[i], 8 * bn_l[i], cudaMemcpyDeviceToDevice, st));
            at += bn_l[i];
        }
        TPZ_CUDA(cudaMemcpyAsync(frow, brow, 8 * u, cudaMemcpyDeviceToDevice, st));
        iota64_kernel<<<grid_for(u), 256, 0, st>>>(bslot, u);
        const int64_t utot = u;
        int64_t h = (int64_t)s.per_key * (kRefineRounds + 1);
        for (int guard = 0; u > 0; ++guard, h *= 2) {
            if (guard > 64) {
                tpz::set_error("tpz_sa_build: internal error (doubling did not finish)");
                return TPZ_E_DEVICE;
            }
            Mem rm(st);
            dbl_key_kernel<<<grid_for(u), 256, 0, st>>>(bidx, u, h, n, isa, key);
            dbl_heads_kernel<<<grid_for(u), 256, 0, st>>>(bgrp, u, head);
            int64_t nseg = 0;
            if ((rc = select_flagged(rm, head, u, hx, dn, &nseg, st))) return rc;
            run_off_kernel<<<grid_for(nseg + 1), 256, 0, st>>>(hx, (int32_t)nseg, u, off);
            // the suffix ids sort with their keys; rows and slots stay in place
            size_t gb = 0;
            TPZ_CUDA(cub::DeviceSegmentedSort::SortPairs(nullptr, gb, key, key2, bidx, t64, (int)u,
                                                         (int)nseg, off, off + 1, st));
            uint8_t *gtmp;
            if ((rc = rm.alloc(&gtmp, gb))) return rc;
            TPZ_CUDA(cub::DeviceSegmentedSort::SortPairs(gtmp, gb, key, key2, bidx, t64, (int)u,
                                                         (int)nseg, off, off + 1, st));
            ++nr;
            TPZ_CUDA(cudaMemcpyAsync(bidx, t64, 8 * u, cudaMemcpyDeviceToDevice, st));
            dbl_mark_kernel<<<grid_for(u), 256, 0, st>>>(bgrp, key2, brow, u, mark);
            size_t sb = 0;
            TPZ_CUDA(cub::DeviceScan::InclusiveScan(nullptr, sb, mark, ng, MaxOp(), u, st));
            uint8_t *stmp;
            if ((rc = rm.alloc(&stmp, sb))) return rc;
            TPZ_CUDA(cub::DeviceScan::InclusiveScan(stmp, sb, mark, ng, MaxOp(), u, st));
            // every key of this round is computed: the ISA may change now
            dbl_update_kernel<<<grid_for(u), 256, 0, st>>>(ng, bidx, brow, bslot, u, isa, fix, keep);
            int64_t u2 = 0;
            if ((rc = select_flagged(rm, keep, u, sel, dn, &u2, st))) return rc;
            if (u2 > 0) dbl_compact_kernel<<<1, 1024, 0, st>>>(sel, u2, brow, bidx, ng, bslot, bgrp);
            u = u2;
        }
        // final rows of the doubling list (frow, increasing) and their
        // suffixes (fix); runs of consecutive rows go to the sink together
        std::vector<int64_t> hrow(utot);
        TPZ_CUDA(cudaMemcpyAsync(hrow.data(), frow, 8 * utot, cudaMemcpyDeviceToHost, st));
        TPZ_CUDA(cudaStreamSynchronize(st));
        for (int64_t a = 0; a < utot;) {
            int64_t b = a + 1;
            while (b < utot && hrow[b] == hrow[b - 1] + 1) ++b;
            if ((rc = em.emit(fix + a, hrow[a], b - a, st))) return rc;
            a = b;
        }
    }
    TPZ_CUDA(cudaGetLastError());
    TPZ_CUDA(cudaStreamSynchronize(st));
    if (rounds) *rounds = nr;
    return TPZ_OK;
}

extern "C" int tpz_sa_build(const uint8_t *T, int64_t n, int64_t *SA, int32_t *rounds) {
    if (n < 0 || (n > 0 && (!T || !SA))) {
        tpz::set_error("tpz_sa_build: bad arguments");
        return TPZ_E_ARG;
    }
    return tpz_sa_build_sink(T, n, host_sink_copy, SA, 0, rounds);
}
