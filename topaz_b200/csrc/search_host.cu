// search_host.cu -- index residency and the host side of the search C ABI.
#include <math.h>
#include <stddef.h>
#include <stdio.h>
#include <string.h>
#include <sys/time.h>

#include <algorithm>
#include <string>
#include <thread>
#include <vector>

#include "search_internal.cuh"

using tpz::search::Cursor;
using tpz::search::DevIndex;
using tpz::search::Hit;
using tpz::search::PopRec;
using tpz::search::QueryOut;

struct tpz_index {
    int dev = 0;
    DevIndex d;
    std::vector<void *> mem;
    int64_t bytes = 0;
    std::vector<int64_t> pstart;   // host copy, Psize + 1
};

namespace {

constexpr char kInternalToAA[] = "ACMLJIVTSKRQZEDBNHYFWXP*G";
constexpr char kMatrixOrder[] = "ARNDCQEGHILKMFPSTWYVBJZX*";

// internal alphabet byte -> matrix index (aa_table2, src/lexicographical.h:19-33)
void internal_map(int8_t out[128]) {
    for (int i = 0; i < 128; ++i) out[i] = 23;
    for (int i = 0; i < 25; ++i) {
        const int m = (int)(strchr(kMatrixOrder, kInternalToAA[i]) - kMatrixOrder);
        out['A' + i] = (int8_t)m;
        out['a' + i] = (int8_t)m;
    }
}

// 25x25 substitution table indexed by internal letters (subject row, query col)
void internal_sub(const int8_t *mat, int8_t out[625]) {
    int8_t m[128];
    internal_map(m);
    for (int t = 0; t < 25; ++t)
        for (int q = 0; q < 25; ++q) out[t * 25 + q] = mat[m['A' + t] * 25 + m['A' + q]];
}

int dalloc(tpz_index *ix, void **p, size_t bytes) {
    TPZ_CUDA(cudaMalloc(p, bytes));
    ix->mem.push_back(*p);
    ix->bytes += (int64_t)bytes;
    return TPZ_OK;
}

// Per-call device buffers, stream-ordered on the calling thread's default
// stream (the library is built with per-thread default streams), so calls
// from different host threads neither wait for each other's allocations nor
// for each other's kernels.  The pool keeps freed memory for the next call
// (tpz::keep_pool_memory).
using tpz::keep_pool_memory;

struct DevBuf {
    std::vector<void *> ptrs;
    DevBuf() { keep_pool_memory(); }
    ~DevBuf() { for (void *p : ptrs) cudaFreeAsync(p, cudaStreamPerThread); }
    template <class T>
    int alloc(T **p, size_t count) {
        void *q = nullptr;
        TPZ_CUDA(cudaMallocAsync(&q, std::max<size_t>(count * sizeof(T), 16), cudaStreamPerThread));
        ptrs.push_back(q);
        *p = (T *)q;
        return TPZ_OK;
    }
};

// bit 1 of *bad: an SA entry outside [0, Tsize); bit 2: a text byte that is
// neither '\n' nor an internal-alphabet letter
__global__ void sa_range_check_kernel(const int64_t *SA, int64_t Tsize, int *bad) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < Tsize;
         i += (int64_t)gridDim.x * blockDim.x)
        if (SA[i] < 0 || SA[i] >= Tsize) atomicOr(bad, 1);
}

__global__ void text_check_kernel(const uint8_t *T, int64_t Tsize, int *bad) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < Tsize;
         i += (int64_t)gridDim.x * blockDim.x) {
        const uint8_t c = T[i];
        if (c != '\n' && (c < 'A' || c > 'Y')) atomicOr(bad, 2);
    }
}

// Host -> device copy of pageable memory (the .psq and .SA file mappings):
// host threads copy 32 MB pieces into two pinned buffers in turn -- touching
// the mapping's pages in parallel -- while the previous piece is on its way
// to the device.  The pinned buffers are made once per index and serve both
// files (pinning memory costs about as much as copying it).
struct UploadStage {
    static constexpr size_t kPiece = 32ull << 20;
    uint8_t *pin[2] = {nullptr, nullptr};
    cudaEvent_t done[2] = {nullptr, nullptr};
    int init() {
        for (int b = 0; b < 2; ++b)
            if (cudaHostAlloc((void **)&pin[b], kPiece, cudaHostAllocDefault) != cudaSuccess ||
                cudaEventCreateWithFlags(&done[b], cudaEventDisableTiming) != cudaSuccess)
                return tpz::cuda_fail(cudaGetLastError(), "index upload buffers");
        return TPZ_OK;
    }
    ~UploadStage() {
        for (int b = 0; b < 2; ++b) {
            if (done[b]) cudaEventDestroy(done[b]);
            if (pin[b]) cudaFreeHost(pin[b]);
        }
    }
};

int upload_pageable(UploadStage &stg, void *dst, const void *src, size_t n) {
    constexpr size_t kPiece = UploadStage::kPiece;
    cudaStream_t st = cudaStreamPerThread;
    int rc = TPZ_OK;
    const unsigned nt = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const uint8_t *s8 = (const uint8_t *)src;
    for (size_t off = 0, k = 0; rc == TPZ_OK && off < n; off += kPiece, ++k) {
        const size_t len = std::min(kPiece, n - off);
        uint8_t *buf = stg.pin[k & 1];
        // the buffer's previous piece (of this or the other file) has left
        if (cudaEventSynchronize(stg.done[k & 1]) != cudaSuccess) {
            rc = tpz::cuda_fail(cudaGetLastError(), "index upload");
            break;
        }
        const size_t part = (len + nt - 1) / nt;
        std::vector<std::thread> th;
        for (unsigned t = 1; t < nt && (size_t)t * part < len; ++t) {
            const size_t a = (size_t)t * part, e = std::min(len, a + part);
            th.emplace_back([=] { memcpy(buf + a, s8 + off + a, e - a); });
        }
        memcpy(buf, s8 + off, std::min(len, part));
        for (std::thread &x : th) x.join();
        if (cudaMemcpyAsync((uint8_t *)dst + off, buf, len, cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaEventRecord(stg.done[k & 1], st) != cudaSuccess)
            rc = tpz::cuda_fail(cudaGetLastError(), "index upload");
    }
    if (cudaStreamSynchronize(st) != cudaSuccess && rc == TPZ_OK)
        rc = tpz::cuda_fail(cudaGetLastError(), "index upload");
    return rc;
}

struct PackArgs {
    const Hit *hits;        // nq * max_cap
    const QueryOut *qout;
    const int64_t *hit_off; // nq + 1
    const int64_t *qoff;
    const int32_t *qlen;
    const int64_t *pstart;
    int nq, max_cap;
    int32_t *protein, *gs, *gl, *so, *sw_status;
    // SW pairs
    int64_t *pq_off, *ps_off;
    int32_t *pq_len, *ps_len, *p_hit;
    const int64_t *pair_off;  // nq + 1: the SW pairs of query q start at pair_off[q]
};

// SW pairs (hits with gapless score >= 40) per query
__global__ void count_pairs_kernel(PackArgs a, int32_t *cnt) {
    __shared__ int c;
    const int q = blockIdx.x;
    const int n = a.qout[q].nhits;
    if (threadIdx.x == 0) c = 0;
    __syncthreads();
    int mine = 0;
    for (int h = threadIdx.x; h < n; h += blockDim.x)
        mine += a.hits[(int64_t)q * a.max_cap + h].gapless_score >= 40;
    if (mine) atomicAdd(&c, mine);
    __syncthreads();
    if (threadIdx.x == 0) cnt[q] = c;
}

// packs the per-query hit lists and lists the SW pairs (gapless >= 40),
// the pairs of a query together
__global__ void pack_hits_kernel(PackArgs a) {
    __shared__ int k0;
    const int q = blockIdx.x;
    const int n = a.qout[q].nhits;
    const int64_t base = a.hit_off[q];
    if (threadIdx.x == 0) k0 = 0;
    __syncthreads();
    for (int h = threadIdx.x; h < n; h += blockDim.x) {
        const Hit x = a.hits[(int64_t)q * a.max_cap + h];
        const int64_t o = base + h;
        a.protein[o] = x.protein;
        a.gs[o] = x.gapless_score;
        a.gl[o] = x.gapless_length;
        a.so[o] = x.suffix_offset;
        if (x.gapless_score < 40) {
            a.sw_status[o] = TPZ_SW_GAPLESS_LOW;
        } else {
            const int64_t k = a.pair_off[q] + atomicAdd(&k0, 1);
            a.pq_off[k] = a.qoff[q];
            a.pq_len[k] = a.qlen[q];
            a.ps_off[k] = a.pstart[x.protein];
            a.ps_len[k] = (int32_t)(a.pstart[x.protein + 1] - a.pstart[x.protein] - 1);
            a.p_hit[k] = (int32_t)o;
        }
    }
}

// sum of qlen * slen over the SW pairs
__global__ void pair_cells_kernel(int64_t n, const int32_t *ql, const int32_t *sl,
                                  unsigned long long *cells) {
    unsigned long long c = 0;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n;
         k += (int64_t)gridDim.x * blockDim.x)
        c += (unsigned long long)ql[k] * (unsigned long long)sl[k];
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xFFFFFFFFu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(cells, c);
}

// SW results of pair k back to hit p_hit[k]; hit2pair (optional) records k
__global__ void scatter_sw_kernel(int64_t n, const int32_t *p_hit, const int32_t *sc,
                                  const int32_t *re, const int32_t *rd, const int32_t *st,
                                  int32_t *raw, int32_t *send, int32_t *qend, int32_t *sw_status,
                                  int32_t *hit2pair) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int h = p_hit[k];
        raw[h] = sc[k];
        send[h] = re[k];
        qend[h] = rd[k];
        sw_status[h] = st[k];
        if (hit2pair) hit2pair[h] = (int32_t)k;
    }
}

// Pairs of the selected (reported) aligned hits, for the SW pass that finds
// their end coordinates after a score-only pass over every hit.
struct SelPairArgs {
    const int32_t *sel, *nsel, *sw_status, *hit2pair;
    int nq, top;
    const int64_t *pq_off, *ps_off;
    const int32_t *pq_len, *ps_len;
    int64_t *lq_off, *ls_off;
    int32_t *lq_len, *ls_len, *lhit, *count;
};

__global__ void selected_pairs_kernel(SelPairArgs a) {
    const int64_t total = (int64_t)a.nq * a.top;
    for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < total;
         x += (int64_t)gridDim.x * blockDim.x) {
        const int q = (int)(x / a.top), t = (int)(x % a.top);
        if (t >= a.nsel[q]) continue;
        const int h = a.sel[x];
        if (a.sw_status[h] != TPZ_SW_OK) continue;
        const int k = a.hit2pair[h];
        const int slot = atomicAdd(a.count, 1);
        a.lq_off[slot] = a.pq_off[k]; a.lq_len[slot] = a.pq_len[k];
        a.ls_off[slot] = a.ps_off[k]; a.ls_len[slot] = a.ps_len[k];
        a.lhit[slot] = h;
    }
}

// ---- report mode: output_top_hits (src/engine.c:193-248) on the device

constexpr int kRawRanks = 32768;      // SW scores 0..32766 (32767 is dropped)
constexpr int kRankThreads = 512;
constexpr int kRankSmemKeys = 16384;  // sort buffer in shared memory up to this size

struct RankArgs {
    const int64_t *hit_off;           // nq + 1
    const int32_t *raw, *sw_status;
    const int32_t *rank_of_raw;       // kRawRanks: dense rank of each score's bitscore
    int32_t rank_low;                 // rank of bitscore 0 (gapless score < 40)
    int low_last;                     // every SW score ranks above bitscore 0
    int low_pass;                     // E-value 1000 passes the cut
    const int32_t *rank_min;          // nq: lowest rank whose E-value passes
    int nq, top, npad;
    uint64_t *gbuf;                   // nq * npad, when the buffer is not in shared memory
    int32_t *sel, *nsel;              // nq * top hit indices in rank order; counts
};

// sort key: bitscore rank descending, then traversal index ascending (the
// stable merge sort of the reference's qsort); bit 0 marks gapless-low hits
__device__ __forceinline__ uint64_t rank_key(int rank, int i, int low) {
    return ((uint64_t)(rank + 1) << 40) | ((uint64_t)(0x7FFFFFFF - i) << 1) | (uint64_t)low;
}

// One block per query: sort the query's aligned hits, keep the first `top`,
// drop those over the E-value cut.
__global__ void __launch_bounds__(kRankThreads) rank_select_kernel(RankArgs a) {
    extern __shared__ uint64_t sbuf[];
    __shared__ int cnt;
    const int q = blockIdx.x;
    uint64_t *buf = a.gbuf ? a.gbuf + (size_t)q * a.npad : sbuf;
    const int64_t base = a.hit_off[q];
    const int n = (int)(a.hit_off[q + 1] - base);
    if (threadIdx.x == 0) cnt = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int st = a.sw_status[base + i];
        uint64_t key = 0;
        if (st == TPZ_SW_OK) key = rank_key(a.rank_of_raw[a.raw[base + i]], i, 0);
        else if (st == TPZ_SW_GAPLESS_LOW && !a.low_last) key = rank_key(a.rank_low, i, 1);
        if (key) buf[atomicAdd(&cnt, 1)] = key;
    }
    __syncthreads();
    const int m = cnt;
    int p = 1;
    while (p < m) p <<= 1;
    for (int i = m + threadIdx.x; i < p; i += blockDim.x) buf[i] = 0;
    __syncthreads();
    // bitonic sort, descending (keys are distinct; padding 0 sorts last)
    for (int k = 2; k <= p; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < p; i += blockDim.x) {
                const int l = i ^ j;
                if (l > i) {
                    const uint64_t x = buf[i], y = buf[l];
                    if (((i & k) == 0) ? (x < y) : (x > y)) { buf[i] = y; buf[l] = x; }
                }
            }
            __syncthreads();
        }
    }
    if (threadIdx.x == 0) {
        int32_t *out = a.sel + (int64_t)q * a.top;
        int ns = 0;
        const int take = min(m, a.top);
        for (int t = 0; t < take; ++t) {
            const uint64_t key = buf[t];
            const int i = 0x7FFFFFFF - (int)((key >> 1) & 0x7FFFFFFF);
            const int rank = (int)(key >> 40) - 1;
            const bool pass = (key & 1) ? a.low_pass != 0 : rank >= a.rank_min[q];
            if (pass) out[ns++] = (int32_t)(base + i);
        }
        if (a.low_last && a.low_pass) {
            // gapless-low hits rank after every aligned hit, in traversal order
            int room = a.top - take;
            for (int i = 0; i < n && room > 0; ++i)
                if (a.sw_status[base + i] == TPZ_SW_GAPLESS_LOW) { out[ns++] = (int32_t)(base + i); --room; }
        }
        a.nsel[q] = ns;
    }
}

// exclusive prefix sum of n counts into off[0..n] (one block of 1024)
__global__ void __launch_bounds__(1024) offsets_kernel(const int32_t *cnt, int n, int64_t *off) {
    __shared__ int64_t part[1024];
    __shared__ int64_t carry;
    const int t = threadIdx.x;
    if (t == 0) carry = 0;
    __syncthreads();
    for (int b = 0; b < n; b += 1024) {
        const int i = b + t;
        const int64_t v = i < n ? cnt[i] : 0;
        part[t] = v;
        __syncthreads();
        for (int o = 1; o < 1024; o <<= 1) {
            const int64_t x = t >= o ? part[t - o] : 0;
            __syncthreads();
            part[t] += x;
            __syncthreads();
        }
        if (i < n) off[i] = carry + part[t] - v;
        __syncthreads();
        if (t == 1023) carry += part[1023];
        __syncthreads();
    }
    if (t == 0) off[n] = carry;
}

constexpr int kGatherFields = 8;
struct GatherArgs {
    const int32_t *sel, *nsel;
    const int64_t *off;
    int nq, top;
    const int32_t *src[kGatherFields];
    int32_t *dst[kGatherFields];
};

__global__ void gather_selected_kernel(GatherArgs g) {
    const int64_t total = (int64_t)g.nq * g.top;
    for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < total;
         x += (int64_t)gridDim.x * blockDim.x) {
        const int q = (int)(x / g.top), k = (int)(x % g.top);
        if (k >= g.nsel[q]) continue;
        const int h = g.sel[x];
        const int64_t d = g.off[q] + k;
#pragma unroll
        for (int f = 0; f < kGatherFields; ++f) g.dst[f][d] = g.src[f][h];
    }
}

struct ResultHolder {
    tpz_search_result r{};
    std::vector<int64_t> hit_off, npops, ncounted, trace_n, trace_row;
    std::vector<int32_t> status, protein, gs, gl, so, raw, qend, send, sw_status;
    std::vector<int32_t> trace_off, trace_score, trace_len, trace_counted;
    std::vector<double> bits, evalue;
    std::vector<int32_t> st_qstart, st_sstart, st_length, st_gapopen, st_mismatch;
    std::vector<double> st_identity;
    int64_t sw_pairs = 0, sw_cells = 0;
    int64_t chain_elems = 0, refill_elems = 0;
};

// Ranking tables of report mode.  The bitscore of a raw score does not
// depend on the query (src/ssw_wrapper.c:179-182), so sorting hits by
// bitscore is sorting them by the dense rank of their score's bitscore; the
// E-value cut of a query is a lowest passing rank, found by bisection since
// the E-value does not increase with the bitscore.
struct RankTables {
    std::vector<int32_t> rank_of_raw;   // kRawRanks
    int32_t rank_low = 0;
    int low_last = 0, low_pass = 0;
    std::vector<int32_t> reps, rep_raw; // ranks held by some raw score (ascending), one raw each
};

int rank_tables(const tpz_search_opts *o, RankTables *t) {
    std::vector<double> b(kRawRanks);
    double ev;
    for (int r = 0; r < kRawRanks; ++r) {
        tpz_karlin(1, 1, 1, o->lambda, o->k, o->H, r, &b[r], &ev);
        if (b[r] != b[r]) { tpz::set_error("tpz_search_batch: bitscores are NaN (check lambda, k)"); return TPZ_E_ARG; }
        // two scores sharing a bitscore must share the E-value too (the cut
        // is taken per rank)
        if (r > 0 && b[r] == b[r - 1] && o->lambda * r - log(o->k) != o->lambda * (r - 1) - log(o->k)) {
            tpz::set_error("tpz_search_batch: lambda too small to rank scores by bitscore");
            return TPZ_E_ARG;
        }
    }
    std::vector<double> u(b);
    u.push_back(0.0);
    std::sort(u.begin(), u.end());
    u.erase(std::unique(u.begin(), u.end()), u.end());
    auto rank = [&](double v) { return (int32_t)(std::lower_bound(u.begin(), u.end(), v) - u.begin()); };
    t->rank_of_raw.resize(kRawRanks);
    std::vector<int32_t> rep(u.size(), -1);
    int32_t minr = INT32_MAX;
    for (int r = 0; r < kRawRanks; ++r) {
        const int32_t k = rank(b[r]);
        t->rank_of_raw[r] = k;
        if (rep[k] < 0) rep[k] = r;
        minr = std::min(minr, k);
    }
    for (size_t k = 0; k < rep.size(); ++k)
        if (rep[k] >= 0) { t->reps.push_back((int32_t)k); t->rep_raw.push_back(rep[k]); }
    t->rank_low = rank(0.0);
    t->low_last = t->rank_low < minr;
    t->low_pass = 1000.0 <= o->max_evalue;
    return TPZ_OK;
}

// lowest rank whose E-value passes for a query of length qlen (INT32_MAX: none)
int32_t rank_min_for(const RankTables &t, const tpz_search_opts *o, int32_t qlen) {
    int64_t lo = 0, hi = (int64_t)t.reps.size();
    while (lo < hi) {
        const int64_t mid = lo + (hi - lo) / 2;
        double bits, ev;
        tpz_karlin(qlen, o->db_size, o->db_proteins, o->lambda, o->k, o->H,
                   t.rep_raw[mid], &bits, &ev);
        if (ev <= o->max_evalue) hi = mid; else lo = mid + 1;
    }
    return lo < (int64_t)t.reps.size() ? t.reps[lo] : INT32_MAX;
}

bool letters_ok(const char *s, int64_t n) {
    for (int64_t i = 0; i < n; ++i)
        if (s[i] < 'A' || s[i] > 'Y') return false;
    return true;
}

// Report mode after the SW of a batch: rank, select and gather on the device,
// then copy the reported hits and score them with tpz_karlin.
struct HitPairs {                 // the SW pairs of a batch and where they came from
    const int8_t *q, *T;
    const int64_t *pq_off, *ps_off;
    const int32_t *pq_len, *ps_len, *hit2pair;
    const int8_t *xmap;           // host, 128 entries
    const int64_t *qoff_q;        // device: text offset of each query
    const int64_t *pstart;        // device: text offset of each protein
};

int report_select(DevBuf &b, ResultHolder *R, int64_t nq, int64_t maxq, const int32_t *qlen,
                  const tpz_search_opts *o, const RankTables &rt, int64_t nh, int32_t *pprot,
                  int32_t *pgs, int32_t *pgl, int32_t *pso, int32_t *raw, int32_t *qend,
                  int32_t *send, int32_t *psw, const HitPairs &hp, cudaEvent_t done) {
    const int top = o->report_hits;
    int npad = 1;
    while (npad < maxq) npad <<= 1;
    std::vector<int32_t> rmin(nq);
    for (int64_t q = 0; q < nq; ++q) rmin[q] = rank_min_for(rt, o, qlen[q]);
    int32_t *d_rank, *d_rmin, *d_sel, *d_nsel; int64_t *d_off, *d_hoff; uint64_t *d_gbuf = nullptr;
    int32_t *dst[kGatherFields];
    int rc;
    if ((rc = b.alloc(&d_rank, kRawRanks)) || (rc = b.alloc(&d_rmin, nq)) ||
        (rc = b.alloc(&d_sel, (size_t)nq * top)) || (rc = b.alloc(&d_nsel, nq)) ||
        (rc = b.alloc(&d_off, nq + 1)) || (rc = b.alloc(&d_hoff, nq + 1)))
        return rc;
    for (int f = 0; f < kGatherFields; ++f)
        if ((rc = b.alloc(&dst[f], (size_t)std::min<int64_t>(nh, nq * (int64_t)top)))) return rc;
    const bool in_smem = npad <= kRankSmemKeys;
    if (!in_smem && (rc = b.alloc(&d_gbuf, (size_t)nq * npad))) return rc;
    TPZ_CUDA(cudaMemcpy(d_rank, rt.rank_of_raw.data(), 4 * kRawRanks, cudaMemcpyHostToDevice));
    TPZ_CUDA(cudaMemcpy(d_rmin, rmin.data(), 4 * nq, cudaMemcpyHostToDevice));
    TPZ_CUDA(cudaMemcpy(d_hoff, R->hit_off.data(), 8 * (nq + 1), cudaMemcpyHostToDevice));
    RankArgs ra;
    ra.hit_off = d_hoff; ra.raw = raw; ra.sw_status = psw; ra.rank_of_raw = d_rank;
    ra.rank_low = rt.rank_low; ra.low_last = rt.low_last; ra.low_pass = rt.low_pass;
    ra.rank_min = d_rmin; ra.nq = (int)nq; ra.top = top; ra.npad = npad; ra.gbuf = d_gbuf;
    ra.sel = d_sel; ra.nsel = d_nsel;
    const size_t smem = in_smem ? sizeof(uint64_t) * npad : 0;
    if (smem > 48 * 1024)
        TPZ_CUDA(cudaFuncSetAttribute((const void *)rank_select_kernel,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    rank_select_kernel<<<(unsigned)nq, kRankThreads, smem>>>(ra);
    offsets_kernel<<<1, 1024>>>(d_nsel, (int)nq, d_off);
    if (hp.hit2pair) {
        // the SW ran scores only: end coordinates of the reported hits
        const int64_t ns = std::min<int64_t>(nh, nq * (int64_t)top);
        SelPairArgs sp;
        int64_t *lqo, *lso; int32_t *lql, *lsl, *lhit, *lcnt, *lsc, *lre, *lrd, *lst;
        if ((rc = b.alloc(&lqo, ns)) || (rc = b.alloc(&lso, ns)) || (rc = b.alloc(&lql, ns)) ||
            (rc = b.alloc(&lsl, ns)) || (rc = b.alloc(&lhit, ns)) || (rc = b.alloc(&lcnt, 1)) ||
            (rc = b.alloc(&lsc, ns)) || (rc = b.alloc(&lre, ns)) || (rc = b.alloc(&lrd, ns)) ||
            (rc = b.alloc(&lst, ns)))
            return rc;
        TPZ_CUDA(cudaMemset(lcnt, 0, 4));
        sp.sel = d_sel; sp.nsel = d_nsel; sp.sw_status = psw; sp.hit2pair = hp.hit2pair;
        sp.nq = (int)nq; sp.top = top; sp.pq_off = hp.pq_off; sp.ps_off = hp.ps_off;
        sp.pq_len = hp.pq_len; sp.ps_len = hp.ps_len; sp.lq_off = lqo; sp.ls_off = lso;
        sp.lq_len = lql; sp.ls_len = lsl; sp.lhit = lhit; sp.count = lcnt;
        const int64_t tot = nq * (int64_t)top;
        selected_pairs_kernel<<<(unsigned)std::min<int64_t>((tot + 255) / 256, 4096), 256>>>(sp);
        int32_t nsp = 0;
        TPZ_CUDA(cudaMemcpy(&nsp, lcnt, 4, cudaMemcpyDeviceToHost));
        if (nsp > 0) {
            rc = tpz::sw::batch_device_x(nsp, hp.q, lqo, lql, hp.T, lso, lsl, o->mat625, o->gap_open,
                                         o->gap_extend, lsc, lre, lrd, lst, 0, hp.xmap, hp.xmap, 0);
            if (rc) return rc;
            scatter_sw_kernel<<<(unsigned)std::min<int64_t>((nsp + 255) / 256, 4096), 256>>>(
                nsp, lhit, lsc, lre, lrd, lst, raw, send, qend, psw, nullptr);
        }
    }
    GatherArgs g;
    g.sel = d_sel; g.nsel = d_nsel; g.off = d_off; g.nq = (int)nq; g.top = top;
    const int32_t *src[kGatherFields] = {pprot, pgs, pgl, pso, raw, qend, send, psw};
    for (int f = 0; f < kGatherFields; ++f) { g.src[f] = src[f]; g.dst[f] = dst[f]; }
    const int64_t tot = nq * (int64_t)top;
    gather_selected_kernel<<<(unsigned)std::min<int64_t>((tot + 255) / 256, 4096), 256>>>(g);
    TPZ_CUDA(cudaGetLastError());
    TPZ_CUDA(cudaEventRecord(done, 0));
    R->hit_off.assign(nq + 1, 0);
    TPZ_CUDA(cudaMemcpy(R->hit_off.data(), d_off, 8 * (nq + 1), cudaMemcpyDeviceToHost));
    const int64_t n = R->hit_off[nq];
    std::vector<int32_t> *host[kGatherFields] = {&R->protein, &R->gs, &R->gl, &R->so,
                                                 &R->raw, &R->qend, &R->send, &R->sw_status};
    for (int f = 0; f < kGatherFields; ++f) {
        host[f]->resize(n);
        if (n) TPZ_CUDA(cudaMemcpy(host[f]->data(), dst[f], 4 * n, cudaMemcpyDeviceToHost));
    }
    if (o->blasttab_stats && n > 0) {
        // the --blasttab columns of the reported hits, on the device
        std::vector<int32_t> qof(n);
        for (int64_t q = 0; q < nq; ++q)
            for (int64_t h = R->hit_off[q]; h < R->hit_off[q + 1]; ++h) qof[h] = (int32_t)q;
        int32_t *d_qof, *sto[5];
        double *d_id;
        if ((rc = b.alloc(&d_qof, n)) || (rc = b.alloc(&d_id, n))) return rc;
        for (int f = 0; f < 5; ++f)
            if ((rc = b.alloc(&sto[f], n))) return rc;
        TPZ_CUDA(cudaMemcpy(d_qof, qof.data(), 4 * n, cudaMemcpyHostToDevice));
        rc = tpz::stats::reported_stats(n, hp.q, hp.qoff_q, d_qof, hp.T, hp.pstart, dst[0], dst[4],
                                        dst[5], dst[6], dst[7], o->mat625, hp.xmap, o->gap_open,
                                        o->gap_extend, sto[0], sto[1], sto[2], sto[3], sto[4], d_id, 0);
        if (rc) return rc;
        std::vector<int32_t> *sh[5] = {&R->st_qstart, &R->st_sstart, &R->st_length, &R->st_gapopen,
                                       &R->st_mismatch};
        for (int f = 0; f < 5; ++f) {
            sh[f]->resize(n);
            TPZ_CUDA(cudaMemcpy(sh[f]->data(), sto[f], 4 * n, cudaMemcpyDeviceToHost));
        }
        R->st_identity.resize(n);
        TPZ_CUDA(cudaMemcpy(R->st_identity.data(), d_id, 8 * n, cudaMemcpyDeviceToHost));
    }
    R->bits.resize(n);
    R->evalue.resize(n);
    for (int64_t q = 0; q < nq; ++q)
        for (int64_t h = R->hit_off[q]; h < R->hit_off[q + 1]; ++h) {
            if (R->sw_status[h] == TPZ_SW_OK) {
                tpz_karlin(qlen[q], o->db_size, o->db_proteins, o->lambda, o->k, o->H, R->raw[h],
                           &R->bits[h], &R->evalue[h]);
            } else {
                R->bits[h] = 0;
                R->evalue[h] = 1000;
            }
        }
    return TPZ_OK;
}

}  // namespace

extern "C" {

int tpz_index_create(const uint8_t *T, int64_t Tsize, const int64_t *SA, const void *ind,
                     int64_t Psize, tpz_index **out) {
    using namespace tpz::search;
    if (!T || !SA || !ind || !out || Tsize < 1 || Psize < 1 || Psize > INT32_MAX - 1) {
        tpz::set_error("tpz_index_create: bad arguments");
        return TPZ_E_ARG;
    }
    *out = nullptr;
    // .ind must tile T exactly: protein p at [start, start+len) then '\n'
    struct Rec { uint64_t hs, ps; int32_t hl, pl; };
    const Rec *rec = (const Rec *)ind;
    std::vector<int64_t> pstart(Psize + 1);
    int64_t run = 0;
    for (int64_t p = 0; p < Psize; ++p) {
        if ((int64_t)rec[p].ps != run || rec[p].pl < 0 || run + rec[p].pl >= Tsize ||
            T[run + rec[p].pl] != '\n') {
            char buf[160];
            snprintf(buf, sizeof buf, "tpz_index_create: .ind record %lld does not match the text",
                     (long long)p);
            tpz::set_error(buf);
            return TPZ_E_ARG;
        }
        pstart[p] = run;
        run += rec[p].pl + 1;
    }
    if (run != Tsize) {
        tpz::set_error("tpz_index_create: .ind does not cover the text");
        return TPZ_E_ARG;
    }
    pstart[Psize] = Tsize;

    tpz_index *ix = new tpz_index();
    TPZ_CUDA(cudaGetDevice(&ix->dev));
    auto fail = [&](int rc) { tpz_index_destroy(ix); return rc; };
    const int64_t sa_rows = ((Tsize * 8 + 4095) / 4096) * 4096 / 8;
    const int64_t nblocks = (Tsize + 63) / 64;
    uint8_t *dT, *dTbase; int64_t *dSA, *dps, *dlb; uint32_t *dnl;
    int rc;
    // 64 bytes in front of the text and 128 behind it: the windows of the
    // extension kernels read a little past both ends
    if ((rc = dalloc(ix, (void **)&dTbase, Tsize + 192))) return fail(rc);
    dT = dTbase + 64;
    if ((rc = dalloc(ix, (void **)&dSA, sa_rows * 8))) return fail(rc);
    if ((rc = dalloc(ix, (void **)&dps, (Psize + 1) * 8))) return fail(rc);
    if ((rc = dalloc(ix, (void **)&dnl, (nblocks + 1) * 4))) return fail(rc);
    if ((rc = dalloc(ix, (void **)&dlb, (kCodes + 1) * 8))) return fail(rc);
    if (cudaMemset(dTbase, '\n', 64) != cudaSuccess ||
        cudaMemset(dT + Tsize, '\n', 128) != cudaSuccess ||
        cudaMemset(dSA + Tsize, 0, (sa_rows - Tsize) * 8) != cudaSuccess ||
        cudaMemcpy(dps, pstart.data(), (Psize + 1) * 8, cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(tpz::cuda_fail(cudaGetLastError(), "tpz_index_create copies"));
    {
        UploadStage stg;
        if ((rc = stg.init()) || (rc = upload_pageable(stg, dT, T, Tsize)) ||
            (rc = upload_pageable(stg, dSA, SA, Tsize * 8)))
            return fail(rc);
    }
    int *dbad;
    if ((rc = dalloc(ix, (void **)&dbad, 4))) return fail(rc);
    cudaMemset(dbad, 0, 4);
    const int nsm = tpz::sm_count();
    // every text byte must be a letter or '\n' (the prefix table indexes by
    // letter) and every SA entry must index T, before any kernel reads them
    text_check_kernel<<<nsm * 8, 256>>>(dT, Tsize, dbad);
    sa_range_check_kernel<<<nsm * 8, 256>>>(dSA, Tsize, dbad);
    int bad = 0;
    if (cudaMemcpy(&bad, dbad, 4, cudaMemcpyDeviceToHost) != cudaSuccess)
        return fail(tpz::cuda_fail(cudaGetLastError(), "tpz_index_create checks"));
    if (bad & 2) {
        tpz::set_error("tpz_index_create: text byte outside the internal alphabet");
        return fail(TPZ_E_ARG);
    }
    if (bad) {
        tpz::set_error("tpz_index_create: SA entry outside [0, Tsize)");
        return fail(TPZ_E_ARG);
    }
    nl_block_count_kernel<<<nsm * 8, 256>>>(dT, Tsize, nblocks, dnl);
    lb_build_kernel<<<nsm * 8, 256>>>(dT, Tsize, dSA, dlb);
    std::vector<uint32_t> cnt(nblocks + 1, 0);
    if (cudaMemcpy(cnt.data(), dnl, nblocks * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
        return fail(tpz::cuda_fail(cudaGetLastError(), "tpz_index_create tables"));
    uint32_t acc = 0;
    for (int64_t b = 0; b <= nblocks; ++b) {
        const uint32_t c = b < nblocks ? cnt[b] : 0;
        cnt[b] = acc;
        acc += c;
    }
    if (cudaMemcpy(dnl, cnt.data(), (nblocks + 1) * 4, cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(tpz::cuda_fail(cudaGetLastError(), "tpz_index_create nl"));
    ix->d.Tsize = Tsize; ix->d.Psize = Psize; ix->d.sa_rows = sa_rows;
    ix->d.T = dT; ix->d.SA = dSA; ix->d.pstart = dps; ix->d.nl = dnl; ix->d.lb = dlb;
    ix->pstart.swap(pstart);
    *out = ix;
    return TPZ_OK;
}

void tpz_index_destroy(tpz_index *ix) {
    if (!ix) return;
    for (void *p : ix->mem) cudaFree(p);
    delete ix;
}

int64_t tpz_index_device_bytes(const tpz_index *ix) { return ix ? ix->bytes : 0; }

int tpz_sa_search_batch(const tpz_index *ix, const char *pcat, const int64_t *poff,
                        const int32_t *plen, int64_t n, int64_t *idx) {
    if (!ix || n < 0) { tpz::set_error("tpz_sa_search_batch: bad arguments"); return TPZ_E_ARG; }
    if (n == 0) return TPZ_OK;
    int64_t bytes = 0;
    for (int64_t i = 0; i < n; ++i) {
        if (plen[i] < 1 || poff[i] < 0 || !letters_ok(pcat + poff[i], plen[i])) {
            tpz::set_error("tpz_sa_search_batch: pattern must be >= 1 internal letters 'A'..'Y'");
            return TPZ_E_ARG;
        }
        bytes = std::max<int64_t>(bytes, poff[i] + plen[i]);
    }
    DevBuf b;
    uint8_t *dp; int64_t *doff, *dout; int32_t *dlen;
    int rc;
    if ((rc = b.alloc(&dp, bytes)) || (rc = b.alloc(&doff, n)) || (rc = b.alloc(&dout, n)) ||
        (rc = b.alloc(&dlen, n)))
        return rc;
    TPZ_CUDA(cudaMemcpy(dp, pcat, bytes, cudaMemcpyHostToDevice));
    TPZ_CUDA(cudaMemcpy(doff, poff, 8 * n, cudaMemcpyHostToDevice));
    TPZ_CUDA(cudaMemcpy(dlen, plen, 4 * n, cudaMemcpyHostToDevice));
    tpz::search::lower_bound_kernel<<<(unsigned)std::min<int64_t>((n + 255) / 256, 4096), 256>>>(
        ix->d, dp, doff, dlen, n, dout);
    TPZ_CUDA(cudaGetLastError());
    TPZ_CUDA(cudaMemcpy(idx, dout, 8 * n, cudaMemcpyDeviceToHost));
    return TPZ_OK;
}

int tpz_sa_hsp_batch(const tpz_index *ix, const char *qcat, const int64_t *qoff,
                     const int32_t *qlen, int64_t nq, const int32_t *query_of,
                     const int32_t *qoffset, const int64_t *row, int64_t n, const int8_t *mat625,
                     int32_t *score, int32_t *length) {
    if (!ix || nq < 1 || n < 0 || !mat625) { tpz::set_error("tpz_sa_hsp_batch: bad arguments"); return TPZ_E_ARG; }
    if (n == 0) return TPZ_OK;
    int64_t bytes = 0;
    for (int64_t q = 0; q < nq; ++q) {
        if (qlen[q] < 1 || qoff[q] < 0 || !letters_ok(qcat + qoff[q], qlen[q])) {
            tpz::set_error("tpz_sa_hsp_batch: queries must be internal letters 'A'..'Y'");
            return TPZ_E_ARG;
        }
        bytes = std::max<int64_t>(bytes, qoff[q] + qlen[q]);
    }
    for (int64_t i = 0; i < n; ++i)
        if (query_of[i] < 0 || query_of[i] >= nq || qoffset[i] < 0 || qoffset[i] >= qlen[query_of[i]]) {
            tpz::set_error("tpz_sa_hsp_batch: (query, offset) out of range");
            return TPZ_E_ARG;
        }
    int8_t sub[625];
    internal_sub(mat625, sub);
    DevBuf b;
    uint8_t *dq; int64_t *dqo, *drow; int32_t *dql, *dqf, *doff, *dsc, *dln; int8_t *dsub;
    int rc;
    // 64 readable bytes in front of the queries and behind them: hsp_at's
    // windows read a little past both ends
    if ((rc = b.alloc(&dq, bytes + 128)) || (rc = b.alloc(&dqo, nq)) || (rc = b.alloc(&dql, nq)) ||
        (rc = b.alloc(&dqf, n)) || (rc = b.alloc(&doff, n)) || (rc = b.alloc(&drow, n)) ||
        (rc = b.alloc(&dsc, n)) || (rc = b.alloc(&dln, n)) || (rc = b.alloc(&dsub, 625)))
        return rc;
    dq += 64;
    TPZ_CUDA(cudaMemcpy(dq, qcat, bytes, cudaMemcpyHostToDevice));
    TPZ_CUDA(cudaMemcpy(dqo, qoff, 8 * nq, cudaMemcpyHostToDevice));
    TPZ_CUDA(cudaMemcpy(dql, qlen, 4 * nq, cudaMemcpyHostToDevice));
    TPZ_CUDA(cudaMemcpy(dqf, query_of, 4 * n, cudaMemcpyHostToDevice));
    TPZ_CUDA(cudaMemcpy(doff, qoffset, 4 * n, cudaMemcpyHostToDevice));
    TPZ_CUDA(cudaMemcpy(drow, row, 8 * n, cudaMemcpyHostToDevice));
    TPZ_CUDA(cudaMemcpy(dsub, sub, 625, cudaMemcpyHostToDevice));
    tpz::search::hsp_batch_kernel<<<(unsigned)std::min<int64_t>((n + 255) / 256, 4096), 256>>>(
        ix->d, dq, dqo, dql, dqf, doff, drow, n, dsub, dsc, dln);
    TPZ_CUDA(cudaGetLastError());
    TPZ_CUDA(cudaMemcpy(score, dsc, 4 * n, cudaMemcpyDeviceToHost));
    TPZ_CUDA(cudaMemcpy(length, dln, 4 * n, cudaMemcpyDeviceToHost));
    return TPZ_OK;
}

int tpz_sa_search(const tpz_index *db, const char *q, int32_t qlen, int64_t offset, int64_t length,
                  int64_t *idx, int64_t *num_matches, int64_t *last_position) {
    // sa_search's own argument checks and return value (src/search.c:276-278)
    if (idx) *idx = -1;
    const int64_t m = length > 0 ? length : (int64_t)qlen - offset;
    if (!db || !q || db->d.Tsize <= 0 || m <= 0 || offset < 0 || offset + m > qlen) {
        tpz::set_error("tpz_sa_search: empty pattern or index, or span outside the query");
        return -1;
    }
    if (!letters_ok(q + offset, m)) {
        tpz::set_error("tpz_sa_search: pattern must be internal letters 'A'..'Y'");
        return TPZ_E_ARG;
    }
    DevBuf b;
    uint8_t *dp;
    int64_t *dout;
    int rc;
    if ((rc = b.alloc(&dp, m)) || (rc = b.alloc(&dout, 3))) return rc;
    cudaStream_t st = cudaStreamPerThread;
    TPZ_CUDA(cudaMemcpyAsync(dp, q + offset, m, cudaMemcpyHostToDevice, st));
    tpz::search::sa_search_call_kernel<<<1, 1, 0, st>>>(db->d, dp, m, dout);
    TPZ_CUDA(cudaGetLastError());
    int64_t h[3];
    TPZ_CUDA(cudaMemcpyAsync(h, dout, sizeof h, cudaMemcpyDeviceToHost, st));
    TPZ_CUDA(cudaStreamSynchronize(st));
    if (idx) *idx = h[0];
    if (num_matches) *num_matches = h[1];
    if (last_position) *last_position = h[2];
    return 0;
}

int tpz_sa_hsp(const tpz_index *db, const char *q, int32_t qlen, int32_t qoffset, int64_t position,
               const int8_t *mat625, int32_t *gapless_score, int32_t *gapless_length) {
    if (!gapless_score || !gapless_length) {
        tpz::set_error("tpz_sa_hsp: NULL output");
        return TPZ_E_ARG;
    }
    const int64_t qo = 0;
    const int32_t qf = 0;
    return tpz_sa_hsp_batch(db, q, &qo, &qlen, 1, &qf, &qoffset, &position, 1, mat625,
                            gapless_score, gapless_length);
}

int tpz_device_init(void) {
    // the primary context and the device pool settings, so that a caller
    // can pay for them on another thread while it reads its input
    TPZ_CUDA(cudaFree(nullptr));
    tpz::sm_count();
    keep_pool_memory();
    return TPZ_OK;
}

int64_t tpz_search_query_device_bytes(int32_t qlen, const tpz_search_opts *o) {
    using namespace tpz::search;
    if (!o || qlen < 0) return -1;
    // the per-query share of tpz_search_batch's device buffers, with the
    // capacities it sizes them by: cursors with their chain caches, protein
    // caches and queue links per searched position; the hitlist scratch
    // (score-bucket lists, hit slots, the protein hash); the hit records;
    // and, per hit, the Smith-Waterman pair and result arrays
    const int64_t ql = qlen > TPZ_SEARCH_MAX_QLEN ? 0 : qlen;
    const int cap = qlen > 3000 ? (int)(1.5 * o->num_hits) : o->alignments;
    const int64_t npos = std::max<int64_t>(0, ql - o->min_hit_length);
    int hash_size = 16;
    while (hash_size < 2 * (cap + 1)) hash_size <<= 1;
    auto al = [](size_t x) { return (int64_t)((x + 15) & ~(size_t)15); };
    const size_t ns = (size_t)cap + 1;
    const int64_t per_q = 7 * al(4 * ns) + 2 * al(4 * (size_t)kSMax) + al(8 * (kSMax / 64)) +
                          2 * al(4 * (size_t)hash_size);
    const int64_t per_pos = 2 * ((int64_t)sizeof(Cursor) + 4 + 2 * 4 * kChain);
    const int64_t per_hit = (int64_t)sizeof(Hit) + 2 * 8 + 18 * 4;
    return (int64_t)qlen + per_q + npos * per_pos + (int64_t)cap * per_hit + 256;
}

int tpz_search_batch(const tpz_index *ix, const char *qcat, const int64_t *qoff,
                     const int32_t *qlen, int64_t nq, const tpz_search_opts *o,
                     tpz_search_result **out) {
    using namespace tpz::search;
    if (!ix || !o || !out || nq < 1 || nq > INT32_MAX / 2 || !o->mat625) {
        tpz::set_error("tpz_search_batch: bad arguments");
        return TPZ_E_ARG;
    }
    *out = nullptr;
    if (!(o->gap_open > o->gap_extend && o->gap_extend >= 0 && o->gap_open <= 255) ||
        o->min_hit_length < 1 || o->seeds < 1 || o->alignments < 1 || o->num_hits < 1 ||
        o->trace_pops < 0) {
        tpz::set_error("tpz_search_batch: invalid options (need 255 >= gap_open > gap_extend >= 0, "
                       "min_hit_length/seeds/alignments/num_hits >= 1)");
        return TPZ_E_ARG;
    }
    const bool report = o->report_hits > 0;
    RankTables rt;
    if (report) {
        if (!(o->k > 0) || o->max_evalue != o->max_evalue) {
            tpz::set_error("tpz_search_batch: report mode needs k > 0 and a max_evalue");
            return TPZ_E_ARG;
        }
        const int rc0 = rank_tables(o, &rt);
        if (rc0) return rc0;
    }
    int maxm = 0;
    for (int i = 0; i < 625; ++i) maxm = std::max<int>(maxm, o->mat625[i]);
    if (255 * maxm >= kSMax) { tpz::set_error("tpz_search_batch: matrix entries too large"); return TPZ_E_ARG; }

    std::vector<int64_t> pos_base(nq + 1, 0), cur_base(nq + 1, 0);
    std::vector<int32_t> qstatus(nq, 0), qlen_eff(nq);
    int64_t bytes = 0;
    int max_cap = 1, max_cursors = 1;
    if (o->ingest < 0 || o->ingest > 2) {
        tpz::set_error("tpz_search_batch: ingest must be 0, 1 or 2");
        return TPZ_E_ARG;
    }
    // raw residues (ingest 1/2) go to the device packed, one query after
    // the other, and are masked and mapped there
    std::vector<char> packed;
    std::vector<int64_t> packed_off;
    if (o->ingest) {
        int64_t tot = 0;
        for (int64_t q = 0; q < nq; ++q) {
            if (qlen[q] < 0 || qoff[q] < 0) {
                tpz::set_error("tpz_search_batch: negative query offset or length");
                return TPZ_E_ARG;
            }
            tot += qlen[q];
        }
        packed.resize(tot + 1);
        packed_off.resize(nq);
        tot = 0;
        for (int64_t q = 0; q < nq; ++q) {
            memcpy(packed.data() + tot, qcat + qoff[q], qlen[q]);
            packed_off[q] = tot;
            tot += qlen[q];
        }
        qcat = packed.data();
        qoff = packed_off.data();
    }
    for (int64_t q = 0; q < nq; ++q) {
        if (qlen[q] < 0 || qoff[q] < 0 || (!o->ingest && !letters_ok(qcat + qoff[q], qlen[q]))) {
            tpz::set_error("tpz_search_batch: queries must be internal letters 'A'..'Y'");
            return TPZ_E_ARG;
        }
        bytes = std::max<int64_t>(bytes, qoff[q] + qlen[q]);
        qlen_eff[q] = qlen[q];
        if (qlen[q] > TPZ_SEARCH_MAX_QLEN) { qstatus[q] |= TPZ_Q_TOO_LONG; qlen_eff[q] = 0; }
        const int64_t np = std::max(0, qlen_eff[q] - o->min_hit_length);
        pos_base[q + 1] = pos_base[q] + np;
        cur_base[q + 1] = 2 * pos_base[q + 1];
        max_cursors = std::max<int>(max_cursors, (int)(2 * np));
        const int cap = qlen[q] > 3000 ? (int)(1.5 * o->num_hits) : o->alignments;
        max_cap = std::max(max_cap, cap);
    }
    const int64_t npos = pos_base[nq];
    int hash_size = 16;
    while (hash_size < 2 * (max_cap + 1)) hash_size <<= 1;
    auto al = [](size_t x) { return (x + 15) & ~(size_t)15; };
    const size_t ns = (size_t)max_cap + 1;
    const size_t per_q = 7 * al(4 * ns) + 2 * al(4 * (size_t)kSMax) + al(8 * (kSMax / 64)) +
                         2 * al(4 * (size_t)hash_size);

    int8_t sub[625], xmap[128];
    internal_sub(o->mat625, sub);
    internal_map(xmap);

    DevBuf b;
    uint8_t *dq, *dscratch; int64_t *dqo, *dpb, *dcb; int32_t *dql, *dqs; int8_t *dsub;
    Cursor *dcur; Hit *dhits; QueryOut *dqout; PopRec *dtrace = nullptr;
    int32_t *dqnext, *dcprot; uint32_t *dcache;
    int rc;
    // 64 readable bytes in front of the queries and behind them: hsp_at's
    // windows read a little past both ends
    if ((rc = b.alloc(&dq, bytes + 128)) || (rc = b.alloc(&dqo, nq)) || (rc = b.alloc(&dql, nq)) ||
        (rc = b.alloc(&dpb, nq + 1)) || (rc = b.alloc(&dcb, nq + 1)) || (rc = b.alloc(&dqs, nq)) ||
        (rc = b.alloc(&dsub, 625)) || (rc = b.alloc(&dcur, 2 * npos + 1)) ||
        (rc = b.alloc(&dscratch, per_q * nq)) || (rc = b.alloc(&dhits, (size_t)nq * max_cap)) ||
        (rc = b.alloc(&dqout, nq)) || (rc = b.alloc(&dqnext, 2 * npos + 1)) ||
        (rc = b.alloc(&dcache, (size_t)kChain * (2 * npos + 1))) ||
        (rc = b.alloc(&dcprot, (size_t)kChain * (2 * npos + 1))))
        return rc;
    dq += 64;
    if (o->trace_pops > 0 && (rc = b.alloc(&dtrace, (size_t)nq * o->trace_pops))) return rc;
    unsigned long long *dqueued;
    if ((rc = b.alloc(&dqueued, 1))) return rc;
    TPZ_CUDA(cudaMemset(dqueued, 0, sizeof(unsigned long long)));
    TPZ_CUDA(cudaMemcpy(dq, qcat, bytes, cudaMemcpyHostToDevice));
    TPZ_CUDA(cudaMemcpy(dqo, qoff, 8 * nq, cudaMemcpyHostToDevice));
    TPZ_CUDA(cudaMemcpy(dql, qlen_eff.data(), 4 * nq, cudaMemcpyHostToDevice));
    TPZ_CUDA(cudaMemcpy(dpb, pos_base.data(), 8 * (nq + 1), cudaMemcpyHostToDevice));
    TPZ_CUDA(cudaMemcpy(dcb, cur_base.data(), 8 * (nq + 1), cudaMemcpyHostToDevice));
    TPZ_CUDA(cudaMemcpy(dqs, qstatus.data(), 4 * nq, cudaMemcpyHostToDevice));
    TPZ_CUDA(cudaMemcpy(dsub, sub, 625, cudaMemcpyHostToDevice));
    if (o->ingest) {
        // SEG (ingest 1) and the internal alphabet on the device; queries
        // past the length limit have length 0 here and stay as they are
        rc = tpz_prepare_queries_device((char *)dq, dqo, dql, nq, bytes, o->ingest == 1, nullptr);
        if (rc) return rc;
    }

    const int nsm = tpz::sm_count();
    struct timeval tw0, tw1;
    gettimeofday(&tw0, nullptr);
    cudaEvent_t ev[5];          // start, walk start, walk end, SW end, seeds done
    for (auto &e : ev) TPZ_CUDA(cudaEventCreate(&e));
    struct EvFree { cudaEvent_t *e; ~EvFree() { for (int i = 0; i < 5; ++i) cudaEventDestroy(e[i]); } } evfree{ev};
    TPZ_CUDA(cudaEventRecord(ev[0], 0));
    if (npos > 0) {
        SeedArgs sa;
        sa.qcat = dq; sa.qoff = dqo; sa.qlen = dql; sa.pos_base = dpb; sa.nq = (int)nq;
        sa.npos = npos; sa.sub = dsub; sa.cursors = dcur; sa.lb_out = nullptr; sa.qstatus = dqs;
        sa.chain = kChain;
        seed_kernel<<<(unsigned)std::min<int64_t>((npos + 127) / 128, (int64_t)nsm * 16), 128>>>(ix->d, sa);
        TPZ_CUDA(cudaEventRecord(ev[4], 0));
        chain_kernel<<<(unsigned)std::min<int64_t>((2 * npos * kChain + 255) / 256, (int64_t)nsm * 64),
                       256>>>(ix->d, sa, o->min_hit_length, dcache, dcprot);
        count_queued_kernel<<<(unsigned)std::min<int64_t>((2 * npos + 255) / 256, (int64_t)nsm * 8), 256>>>(
            dcur, 2 * npos, o->min_hit_length, dqueued);
    }
    WalkArgs wa;
    wa.qcat = dq; wa.qoff = dqo; wa.qlen = dql; wa.nq = (int)nq; wa.cursor_base = dcb;
    wa.cursors = dcur; wa.sub = dsub; wa.min_hit_length = o->min_hit_length;
    wa.seeds = o->seeds; wa.alignments = o->alignments; wa.num_hits = o->num_hits;
    wa.max_cap = max_cap; wa.hash_size = hash_size; wa.max_cursors = max_cursors;
    wa.scratch = dscratch; wa.scratch_per_query = per_q; wa.hits = dhits; wa.qout = dqout;
    wa.qstatus = dqs; wa.trace = dtrace; wa.trace_cap = o->trace_pops;
    wa.qnext = dqnext; wa.ccache = dcache; wa.cprot = dcprot;
    TPZ_CUDA(cudaEventRecord(ev[1], 0));
    walk_kernel<<<(unsigned)((nq + kWalkWarps - 1) / kWalkWarps), kWalkWarps * 32>>>(ix->d, wa);
    TPZ_CUDA(cudaGetLastError());
    TPZ_CUDA(cudaEventRecord(ev[2], 0));

    ResultHolder *R = new ResultHolder();
    std::vector<QueryOut> qo(nq);
    auto bail = [&](int code) { delete R; return code; };
    if (cudaMemcpy(qo.data(), dqout, sizeof(QueryOut) * nq, cudaMemcpyDeviceToHost) != cudaSuccess)
        return bail(tpz::cuda_fail(cudaGetLastError(), "tpz_search_batch walk"));
    R->hit_off.assign(nq + 1, 0);
    R->npops.resize(nq); R->ncounted.resize(nq); R->status.resize(nq);
    {
        unsigned long long queued = 0;
        if (cudaMemcpy(&queued, dqueued, sizeof queued, cudaMemcpyDeviceToHost) != cudaSuccess)
            return bail(tpz::cuda_fail(cudaGetLastError(), "tpz_search_batch counts"));
        int64_t refills = 0;
        for (int64_t q = 0; q < nq; ++q) refills += qo[q].refills;
        R->chain_elems = (int64_t)queued * kChain;
        R->refill_elems = refills * 32;
    }
    for (int64_t q = 0; q < nq; ++q) {
        R->hit_off[q + 1] = R->hit_off[q] + qo[q].nhits;
        R->npops[q] = qo[q].npops;
        R->ncounted[q] = qo[q].ncounted;
        R->status[q] = qo[q].status | qstatus[q];
    }
    const int64_t nh = R->hit_off[nq];
    if (!report)
        for (auto *v : {&R->protein, &R->gs, &R->gl, &R->so, &R->raw, &R->qend, &R->send, &R->sw_status})
            v->assign(nh, -1);
    int64_t maxq = 0;
    for (int64_t q = 0; q < nq; ++q) maxq = std::max<int64_t>(maxq, qo[q].nhits);

    if (nh > 0) {
        int64_t *dho, *pq_off, *ps_off, *dpoff; int32_t *pprot, *pgs, *pgl, *pso, *psw, *pq_len, *ps_len, *p_hit, *dnp;
        int32_t *sc, *re, *rd, *st, *raw, *qend, *send, *hit2pair;
        if ((rc = b.alloc(&dho, nq + 1)) || (rc = b.alloc(&pprot, nh)) || (rc = b.alloc(&pgs, nh)) ||
            (rc = b.alloc(&pgl, nh)) || (rc = b.alloc(&pso, nh)) || (rc = b.alloc(&psw, nh)) ||
            (rc = b.alloc(&pq_off, nh)) || (rc = b.alloc(&ps_off, nh)) || (rc = b.alloc(&pq_len, nh)) ||
            (rc = b.alloc(&ps_len, nh)) || (rc = b.alloc(&p_hit, nh)) || (rc = b.alloc(&dnp, nq)) ||
            (rc = b.alloc(&dpoff, nq + 1)) ||
            (rc = b.alloc(&sc, nh)) || (rc = b.alloc(&re, nh)) || (rc = b.alloc(&rd, nh)) ||
            (rc = b.alloc(&st, nh)) || (rc = b.alloc(&raw, nh)) || (rc = b.alloc(&qend, nh)) ||
            (rc = b.alloc(&send, nh)) || (rc = b.alloc(&hit2pair, report ? nh : 1)))
            return bail(rc);
        if (cudaMemcpy(dho, R->hit_off.data(), 8 * (nq + 1), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemset(raw, 0xFF, 4 * nh) != cudaSuccess ||
            cudaMemset(qend, 0xFF, 4 * nh) != cudaSuccess || cudaMemset(send, 0xFF, 4 * nh) != cudaSuccess)
            return bail(tpz::cuda_fail(cudaGetLastError(), "tpz_search_batch pack"));
        PackArgs pa;
        pa.hits = dhits; pa.qout = dqout; pa.hit_off = dho; pa.qoff = dqo; pa.qlen = dql;
        pa.pstart = ix->d.pstart; pa.nq = (int)nq; pa.max_cap = max_cap;
        pa.protein = pprot; pa.gs = pgs; pa.gl = pgl; pa.so = pso; pa.sw_status = psw;
        pa.pq_off = pq_off; pa.ps_off = ps_off; pa.pq_len = pq_len; pa.ps_len = ps_len;
        pa.p_hit = p_hit; pa.pair_off = dpoff;
        count_pairs_kernel<<<(unsigned)nq, 256>>>(pa, dnp);
        offsets_kernel<<<1, 1024>>>(dnp, (int)nq, dpoff);
        pack_hits_kernel<<<(unsigned)nq, 256>>>(pa);
        std::vector<int64_t> poff(nq + 1);
        if (cudaMemcpy(poff.data(), dpoff, 8 * (nq + 1), cudaMemcpyDeviceToHost) != cudaSuccess)
            return bail(tpz::cuda_fail(cudaGetLastError(), "tpz_search_batch pairs"));
        const int64_t npairs = poff[nq];
        R->sw_pairs = npairs;
        if (npairs > 0) {
            unsigned long long *dcells;
            if ((rc = b.alloc(&dcells, 1))) return bail(rc);
            TPZ_CUDA(cudaMemset(dcells, 0, 8));
            pair_cells_kernel<<<(unsigned)std::min<int64_t>((npairs + 255) / 256, 2048), 256>>>(
                npairs, pq_len, ps_len, dcells);
            unsigned long long cells = 0;
            TPZ_CUDA(cudaMemcpy(&cells, dcells, 8, cudaMemcpyDeviceToHost));
            R->sw_cells = (int64_t)cells;
        }
        if (npairs > 0) {
            // the pairs of a query share its profile; report mode ranks on
            // scores alone (end coordinates come later, for the reported hits)
            rc = tpz::sw::batch_device_grouped(npairs, (const int8_t *)dq, pq_off, pq_len,
                                               (const int8_t *)ix->d.T, ps_off, ps_len, o->mat625,
                                               o->gap_open, o->gap_extend, sc, re, rd, st, 0, xmap,
                                               xmap, report ? 1 : 0, nq, dpoff, poff.data(),
                                               qlen_eff.data());
            if (rc) return bail(rc);
            scatter_sw_kernel<<<(unsigned)std::min<int64_t>((npairs + 255) / 256, 4096), 256>>>(
                npairs, p_hit, sc, re, rd, st, raw, send, qend, psw, report ? hit2pair : nullptr);
        }
        if (report) {
            HitPairs hp;
            hp.q = (const int8_t *)dq; hp.T = (const int8_t *)ix->d.T; hp.pq_off = pq_off;
            hp.ps_off = ps_off; hp.pq_len = pq_len; hp.ps_len = ps_len;
            hp.hit2pair = npairs > 0 ? hit2pair : nullptr; hp.xmap = xmap;
            hp.qoff_q = dqo; hp.pstart = ix->d.pstart;
            int rc2 = report_select(b, R, nq, maxq, qlen, o, rt, nh, pprot, pgs, pgl, pso, raw, qend, send,
                                    psw, hp, ev[3]);
            if (rc2) return bail(rc2);
        } else {
        if (cudaEventRecord(ev[3], 0) != cudaSuccess)
            return bail(tpz::cuda_fail(cudaGetLastError(), "tpz_search_batch event"));
        if (cudaMemcpy(R->protein.data(), pprot, 4 * nh, cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(R->gs.data(), pgs, 4 * nh, cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(R->gl.data(), pgl, 4 * nh, cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(R->so.data(), pso, 4 * nh, cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(R->sw_status.data(), psw, 4 * nh, cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(R->raw.data(), raw, 4 * nh, cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(R->qend.data(), qend, 4 * nh, cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(R->send.data(), send, 4 * nh, cudaMemcpyDeviceToHost) != cudaSuccess)
            return bail(tpz::cuda_fail(cudaGetLastError(), "tpz_search_batch results"));
        }
    } else if (report) {
        R->hit_off.assign(nq + 1, 0);
    }
    if (o->trace_pops > 0) {
        std::vector<PopRec> tr((size_t)nq * o->trace_pops);
        if (cudaMemcpy(tr.data(), dtrace, sizeof(PopRec) * tr.size(), cudaMemcpyDeviceToHost) != cudaSuccess)
            return bail(tpz::cuda_fail(cudaGetLastError(), "tpz_search_batch trace"));
        R->trace_n.resize(nq);
        R->trace_row.resize(tr.size()); R->trace_off.resize(tr.size());
        R->trace_score.resize(tr.size()); R->trace_len.resize(tr.size()); R->trace_counted.resize(tr.size());
        for (size_t i = 0; i < tr.size(); ++i) {
            R->trace_row[i] = tr[i].row; R->trace_off[i] = tr[i].off; R->trace_score[i] = tr[i].score;
            R->trace_len[i] = tr[i].len; R->trace_counted[i] = tr[i].counted;
        }
        for (int64_t q = 0; q < nq; ++q) R->trace_n[q] = std::min<int64_t>(qo[q].npops, o->trace_pops);
    }
    tpz_search_result &r = R->r;
    r.nq = nq; r.nhits_total = nh; r.hit_off = R->hit_off.data(); r.npops = R->npops.data();
    r.ncounted = R->ncounted.data(); r.status = R->status.data(); r.protein = R->protein.data();
    r.gapless_score = R->gs.data(); r.gapless_length = R->gl.data(); r.suffix_offset = R->so.data();
    r.rawscore = R->raw.data(); r.qend = R->qend.data(); r.send = R->send.data();
    r.sw_status = R->sw_status.data();
    r.trace_n = o->trace_pops > 0 ? R->trace_n.data() : nullptr;
    r.trace_row = o->trace_pops > 0 ? R->trace_row.data() : nullptr;
    r.trace_off = o->trace_pops > 0 ? R->trace_off.data() : nullptr;
    r.trace_score = o->trace_pops > 0 ? R->trace_score.data() : nullptr;
    r.trace_len = o->trace_pops > 0 ? R->trace_len.data() : nullptr;
    r.trace_counted = o->trace_pops > 0 ? R->trace_counted.data() : nullptr;
    if (report) {
        r.nhits_total = R->hit_off[nq];
        r.bitscore = R->bits.data();
        r.evalue = R->evalue.data();
        if (o->blasttab_stats) {
            // every reported hit has its columns (none when nothing was reported)
            const int64_t n = R->hit_off[nq];
            R->st_qstart.resize(n); R->st_sstart.resize(n); R->st_length.resize(n);
            R->st_gapopen.resize(n); R->st_mismatch.resize(n); R->st_identity.resize(n);
            r.qstart = R->st_qstart.data(); r.sstart = R->st_sstart.data();
            r.length = R->st_length.data(); r.gapopen = R->st_gapopen.data();
            r.mismatch = R->st_mismatch.data(); r.identity = R->st_identity.data();
        }
    }
    TPZ_CUDA(cudaStreamSynchronize(cudaStreamPerThread));
    float t01 = 0, t12 = 0, t23 = 0;
    cudaEventElapsedTime(&t01, ev[0], ev[1]);
    float t04 = 0;
    if (npos > 0) cudaEventElapsedTime(&t04, ev[0], ev[4]);
    r.seed_ms = t04;
    r.chain_ms = npos > 0 ? t01 - t04 : 0;
    r.positions = npos;
    cudaEventElapsedTime(&t12, ev[1], ev[2]);
    if (nh > 0) cudaEventElapsedTime(&t23, ev[2], ev[3]);
    gettimeofday(&tw1, nullptr);
    r.stage_ms[0] = t01;
    r.stage_ms[1] = t12;
    r.stage_ms[2] = t23;
    r.stage_ms[3] = (tw1.tv_sec - tw0.tv_sec) * 1e3 + (tw1.tv_usec - tw0.tv_usec) / 1e3;
    r.sw_pairs = R->sw_pairs;
    r.sw_cells = R->sw_cells;
    r.chain_elems = R->chain_elems;
    r.refill_elems = R->refill_elems;
    *out = &R->r;
    return TPZ_OK;
}

void tpz_search_result_free(tpz_search_result *r) {
    if (!r) return;
    ResultHolder *h = reinterpret_cast<ResultHolder *>(reinterpret_cast<char *>(r) -
                                                       offsetof(ResultHolder, r));
    delete h;
}

void tpz_karlin(int32_t qlen, uint64_t db_size, uint64_t db_proteins, double lambda, double k,
                double H, int32_t raw, double *bitscore, double *evalue) {
    const double correction = log(k * qlen * db_size) / H;
    const double corrected_q = fmax(qlen - correction, 1.0);
    const double corrected_db = fmax(db_size - (correction * db_proteins), 1.0);
    double bits = (lambda * raw - log(k));
    double ev = corrected_q * corrected_db * exp(-bits);
    ev = ev > 1.0e-180 ? ev : 0.0;
    *bitscore = bits / M_LN2;
    *evalue = ev;
}

}  // extern "C"
