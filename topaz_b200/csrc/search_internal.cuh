// search_internal.cuh -- device structures of the search path.
#pragma once

#include "tpz_common.cuh"

namespace tpz {
namespace search {

constexpr int kK = 5;                       // prefix-table width (symbols)
constexpr int64_t kCodes = 11881376;        // 26^5
constexpr int kSMax = 4352;                 // gapless scores are < 255*17+1 <= kSMax

struct DevIndex {
    int64_t Tsize = 0, Psize = 0, sa_rows = 0;
    const uint8_t *T = nullptr;
    const int64_t *SA = nullptr;
    const int64_t *pstart = nullptr;    // Psize + 1
    const uint32_t *nl = nullptr;       // per 64-byte block
    const int64_t *lb = nullptr;        // kCodes + 1
};

struct Cursor {
    int64_t row;
    int32_t off;
    int16_t dir;
    uint8_t cpos, cn;    // next unused / valid entries of the cursor's element cache
    int32_t score, len;
    int32_t prot;        // protein of the current row
};

constexpr int kWalkWarps = 4;            // queries (warps) per walk block
constexpr int kChain = 64;               // chain elements cached per cursor
static_assert(kChain >= 32, "a walk refill stores 32 chain elements in a cursor's cache slot");

struct Hit {
    int32_t protein, gapless_score, gapless_length, suffix_offset;
};

struct PopRec {
    int64_t row;
    int32_t off, score, len, counted;
};

struct QueryOut {
    int64_t npops, ncounted;
    int32_t nhits, status;
    int64_t refills;              // chain caches the walk refilled (32 elements each)
};

struct SeedArgs {
    const uint8_t *qcat;
    const int64_t *qoff;
    const int32_t *qlen;
    const int64_t *pos_base;   // nq + 1: searched positions before each query
    int nq;
    int64_t npos;
    const int8_t *sub;         // 25x25 by internal letter (subject row, query col)
    Cursor *cursors;           // 2 per position
    int64_t *lb_out;           // optional: bound per position (-2 skipped)
    int32_t *qstatus;          // per query status bits
    int chain;                 // chain elements precomputed per cursor (0 or kChain)
};

struct WalkArgs {
    const uint8_t *qcat;
    const int64_t *qoff;
    const int32_t *qlen;
    int nq;
    const int64_t *cursor_base;   // nq + 1
    Cursor *cursors;
    const int8_t *sub;
    int min_hit_length, seeds, alignments, num_hits;
    int max_cap, hash_size, max_cursors;
    uint8_t *scratch;             // per query: hitlist structures
    size_t scratch_per_query;
    int32_t *qnext;               // per cursor (global cursor index)
    uint32_t *ccache;             // 32 packed chain elements per cursor
    int32_t *cprot;               // the protein of each chain element's row
    Hit *hits;                    // nq * max_cap
    QueryOut *qout;
    const int32_t *qstatus;
    PopRec *trace;                // optional: nq * trace_cap
    int64_t trace_cap;
};

__global__ void nl_block_count_kernel(const uint8_t *T, int64_t Tsize, int64_t nblocks, uint32_t *cnt);
__global__ void lb_build_kernel(const uint8_t *T, int64_t Tsize, const int64_t *SA, int64_t *lb);
__global__ void seed_kernel(DevIndex ix, SeedArgs a);
__global__ void walk_kernel(DevIndex ix, WalkArgs a);
__global__ void chain_kernel(DevIndex ix, SeedArgs a, int min_hit_length, uint32_t *cache,
                             int32_t *cprot);
__global__ void hsp_batch_kernel(DevIndex ix, const uint8_t *qcat, const int64_t *qoff,
                                 const int32_t *qlen, const int32_t *query_of, const int32_t *off,
                                 const int64_t *row, int64_t n, const int8_t *sub, int32_t *score,
                                 int32_t *len);
__global__ void lower_bound_kernel(DevIndex ix, const uint8_t *pcat, const int64_t *poff,
                                   const int32_t *plen, int64_t n, int64_t *out);
__global__ void count_queued_kernel(const Cursor *cursors, int64_t n, int min_hit_length,
                                    unsigned long long *count);
__global__ void sa_search_call_kernel(DevIndex ix, const uint8_t *P, int64_t m, int64_t *out3);

}  // namespace search

namespace sw {
// Batched SW over device buffers; xq/xs (128-entry maps, may be null) turn
// query/subject bytes into matrix indices inside the kernel; score_only
// skips the end coordinates (ref_end = read_end = -2 for TPZ_SW_OK pairs).
int batch_device_x(int64_t n, const int8_t *q, const int64_t *qoff, const int32_t *qlen,
                   const int8_t *s, const int64_t *soff, const int32_t *slen, const int8_t *mat,
                   int go, int ge, int32_t *score, int32_t *ref_end, int32_t *read_end,
                   int32_t *status, cudaStream_t st, const int8_t *xq, const int8_t *xs,
                   int score_only, const int32_t *subset = nullptr, int64_t nsub = 0,
                   int known_multi_maxn = -1, int lane = 0);
// known_multi_maxn >= 0: the caller knows the longest subject among pairs
// with queries longer than one 1,024-row stripe (0: no such pair), so the
// call need not read it back from the device before sizing the stripe
// boundary buffer (no host wait inside the call).  lane 0/1: calls of one
// host thread that run concurrently use different lanes (own streams).
// The same for pairs grouped by query (group g = pairs [gstart[g],
// gstart[g+1]), all with query length gqlen[g]): groups with enough pairs go
// to the query-major kernels, one shared profile per query; the rest by pair.
int batch_device_grouped(int64_t n, const int8_t *q, const int64_t *qoff, const int32_t *qlen,
                         const int8_t *s, const int64_t *soff, const int32_t *slen,
                         const int8_t *mat, int go, int ge, int32_t *score, int32_t *ref_end,
                         int32_t *read_end, int32_t *status, cudaStream_t st, const int8_t *xq,
                         const int8_t *xs, int score_only, int64_t ngroups,
                         const int64_t *gstart_dev, const int64_t *gstart_host,
                         const int32_t *gqlen_host);
}  // namespace sw

namespace stats {
// The --blasttab columns of n reported search hits (stats_kernel.cu): hit d
// of query query_of[d] (text at qtext + qoff_q[query]) against protein
// protein[d] of the index text T (from pstart[protein]), residues mapped by
// xmap; hits whose sw_status is not TPZ_SW_OK get -1 columns.  Waits for
// its work on `st`.
int reported_stats(int64_t n, const int8_t *qtext, const int64_t *qoff_q, const int32_t *query_of,
                   const int8_t *T, const int64_t *pstart, const int32_t *protein,
                   const int32_t *raw, const int32_t *qend, const int32_t *send,
                   const int32_t *sw_status, const int8_t *mat, const int8_t *xmap, int go, int ge,
                   int32_t *qstart, int32_t *sstart, int32_t *length, int32_t *gapopen,
                   int32_t *mismatch, double *identity, cudaStream_t st);
}  // namespace stats

}  // namespace tpz
