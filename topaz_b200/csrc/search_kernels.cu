// search_kernels.cu -- resident index, seed lookup, gapless extension and the
// best-first SA walk with its hitlist, for sm_100a.
//
// Reference path (src/query.c:94-174): for each query position a lower-bound
// search of the query suffix in the suffix array (sa_search), sa_hsp at the
// bound and the row before it, then a best-first walk over adjacent SA rows
// (pqueue_next) feeding a capped hitlist (hitlist_add) until -S counted pops
// or an empty queue.
//
// Device layout of the index (one copy in HBM, built once per DB):
//   T        the .psq bytes (internal alphabet + '\n'), padded with '\n'
//   SA       int64 rows; rows [Tsize, sa_rows) are zero -- the reference
//            mmaps .SA and its reads past the end (search.c:100, hit.c:138
//            with db_valid_index comparing rows against a byte size,
//            db.c:249-251) see the zero fill of the file's last page
//   pstart   protein start offsets (from .ind), Psize + 1 entries
//   nl       number of '\n' before each 64-byte block of T: the protein of a
//            text position is nl[pos/64] + the '\n' bytes in its block before
//            it (db_index, db.c:176-205, counts the delimiter as part of the
//            preceding protein)
//   lb       for each 5-symbol prefix code (26-ary, '\n' = 0, 'A'..'Y' =
//            1..25, symbols after a '\n' read as 0) the number of suffixes
//            whose prefix code is smaller; the rows of a code are
//            [lb[c], lb[c+1]).  Suffix order and prefix-code order agree
//            because '\n' sorts below every letter, so a lower bound needs a
//            binary search only inside one bucket, starting 5 symbols in.
//
// Walk state per query (one thread, exact sequential semantics):
//   the priority queue of suffix cursors is an array of per-score stacks:
//   among equal scores the newest insert pops first, as with rb_popmax on a
//   tree where equal keys go right (rbtree.c:70-78, :410-427);
//   the hitlist keeps per-score FIFO lists (rb_popmin/rb_getmin take the
//   oldest of the smallest score, rbtree.c:429-457; rb_reput re-inserts as
//   newest, :496-505) plus an open-addressing protein -> hit table with
//   backward-shift deletion.

#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "search_internal.cuh"

namespace tpz {
namespace search {

// ---------------------------------------------------------------- helpers

__device__ __forceinline__ int sym(uint8_t c) { return c == '\n' ? 0 : (int)c - 'A' + 1; }

// prefix code of the text suffix at idx (K symbols, zero after a '\n')
__device__ __forceinline__ int64_t text_code(const uint8_t *T, int64_t Tsize, int64_t idx) {
    int64_t code = 0;
    bool ended = false;
#pragma unroll
    for (int i = 0; i < kK; ++i) {
        int d = 0;
        if (!ended) {
            const int64_t p = idx + i;
            const uint8_t c = p < Tsize ? T[p] : (uint8_t)'\n';
            if (c == '\n') ended = true; else d = sym(c);
        }
        code = code * 26 + d;
    }
    return code;
}

// exact count of '\n' bytes in T[base, pos) with base = pos & ~63
__device__ __forceinline__ int newlines_in_block_before(const uint8_t *T, int64_t pos) {
    const int64_t base = pos & ~(int64_t)63;
    const int n = (int)(pos - base);
    const uint64_t *w = reinterpret_cast<const uint64_t *>(T + base);
    int cnt = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        if (8 * i >= n) break;
        const uint64_t x = __ldg(w + i) ^ 0x0A0A0A0A0A0A0A0Aull;
        uint64_t y = (x & 0x7F7F7F7F7F7F7F7Full) + 0x7F7F7F7F7F7F7F7Full;
        y = ~(y | x | 0x7F7F7F7F7F7F7F7Full);      // 0x80 in every byte that was '\n'
        const int keep = n - 8 * i;                   // bytes of this word before pos
        if (keep < 8) y &= (1ull << (8 * keep)) - 1;
        cnt += __popcll(y);
    }
    return cnt;
}

__device__ __forceinline__ int64_t protein_of(const DevIndex &ix, int64_t pos) {
    return (int64_t)ix.nl[pos >> 6] + newlines_in_block_before(ix.T, pos);
}

// 32 bytes of memory from p (any alignment) as 8 words in memory order:
// nine aligned 4-byte loads issued together, funnel-shifted into place, so
// the window stays in registers.  Reads up to 3 bytes before p and 35 after
// it: the text and query buffers keep 64 readable bytes in front of their
// first byte and behind their last.
__device__ __forceinline__ void load32(const uint8_t *p, uint32_t (&w)[8]) {
    const uintptr_t a = (uintptr_t)p & ~(uintptr_t)3;
    const uint32_t sh = (uint32_t)((uintptr_t)p - a) * 8u;
    const uint32_t *src = reinterpret_cast<const uint32_t *>(a);
    uint32_t r[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) r[k] = __ldg(src + k);
#pragma unroll
    for (int k = 0; k < 8; ++k) w[k] = __funnelshift_r(r[k], r[k + 1], sh);
}

// byte k (a compile-time index after unrolling) of a load32 window
__device__ __forceinline__ uint32_t byte_of(const uint32_t (&w)[8], int k) {
    return (w[k >> 2] >> (8 * (k & 3))) & 0xFFu;
}

// sa_hsp (src/search.c:99-190) at text position idx for query offset off.
// Returns the length (-1 when the first symbols differ; score untouched then).
// The windows (up to 128 bytes each side) are read 32 bytes per round trip
// into registers; the running sums walk them in the reference's order and
// stop at the first '\n' exactly as its byte loop does.
__device__ int hsp_at(const DevIndex &ix, int64_t idx, const uint8_t *Q, int qlen, int off,
                      const int8_t *sub, int *score) {
    const uint8_t *t = ix.T + idx;
    const uint8_t *q = Q + off;
    int64_t mr = ix.Tsize - idx;
    if (mr > qlen - off) mr = qlen - off;
    if (mr > 128) mr = 128;
    uint32_t tw[8], qw[8];
    load32(t, tw);
    load32(q, qw);
    if ((tw[0] & 0xFFu) != (qw[0] & 0xFFu)) return -1;
    int run = 0, best_r = 0, arg_r = 0;
    bool stop = false;
    for (int i0 = 0; i0 < (int)mr && !stop; i0 += 32) {
        if (i0 > 0) { load32(t + i0, tw); load32(q + i0, qw); }
#pragma unroll
        for (int k = 0; k < 32; ++k) {
            const uint32_t c = byte_of(tw, k);
            if (!stop && i0 + k < (int)mr) {
                if (c == '\n') {
                    stop = true;
                } else {
                    run += sub[(c - 'A') * 25 + (byte_of(qw, k) - 'A')];
                    if (run >= best_r) { best_r = run; arg_r = i0 + k; }
                }
            }
        }
    }
    int64_t ml = idx < off ? idx : off;
    if (ml > 128) ml = 128;
    int best_l = 0, arg_l = 0;
    run = 0;
    stop = false;
    // left: i = 1 .. ml-1 reads t[-i]; a round loads the 32 bytes that end at
    // t[-i0], so t[-(i0 + k)] is byte 31 - k
    for (int i0 = 1; i0 < (int)ml && !stop; i0 += 32) {
        load32(t - (i0 + 31), tw);
        load32(q - (i0 + 31), qw);
#pragma unroll
        for (int k = 0; k < 32; ++k) {
            const uint32_t c = byte_of(tw, 31 - k);
            if (!stop && i0 + k < (int)ml) {
                if (c == '\n') {
                    stop = true;
                } else {
                    run += sub[(c - 'A') * 25 + (byte_of(qw, 31 - k) - 'A')];
                    if (run >= best_l) { best_l = run; arg_l = i0 + k; }
                }
            }
        }
    }
    *score = best_l + best_r;
    return arg_l + arg_r;
}

// lower bound of the suffix P[0, m) (letters only) over the whole SA
__device__ int64_t lower_bound(const DevIndex &ix, const uint8_t *P, int m) {
    int64_t code = 0;
    const int kk = m < kK ? m : kK;
#pragma unroll
    for (int i = 0; i < kK; ++i) code = code * 26 + (i < kk ? sym(P[i]) : 0);
    int64_t lo = ix.lb[code];
    if (m <= kK) return lo;        // exact: every suffix with this prefix is >= P
    int64_t hi = ix.lb[code + 1];
    while (lo < hi) {
        const int64_t mid = lo + ((hi - lo) >> 1);
        const int64_t s = ix.SA[mid] + kK;
        // compare T[s..] with P[kK..]
        int r = 0;
        int64_t i = s;
        int j = kK;
        for (;;) {
            if (j == m) { r = 0; break; }                 // P is a prefix: not less
            if (i >= ix.Tsize) { r = -1; break; }          // text ended first: less
            const int d = (int)ix.T[i] - (int)P[j];
            if (d) { r = d; break; }
            ++i; ++j;
        }
        if (r < 0) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// ---------------------------------------------------------- index build

__global__ void nl_block_count_kernel(const uint8_t *T, int64_t Tsize, int64_t nblocks,
                                      uint32_t *cnt) {
    for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < nblocks;
         b += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t *w = reinterpret_cast<const uint64_t *>(T + 64 * b);
        int c = 0;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const uint64_t x = w[i] ^ 0x0A0A0A0A0A0A0A0Aull;
            uint64_t y = (x & 0x7F7F7F7F7F7F7F7Full) + 0x7F7F7F7F7F7F7F7Full;
            y = ~(y | x | 0x7F7F7F7F7F7F7F7Full);
            c += __popcll(y);
        }
        cnt[b] = c;   // includes pad bytes past Tsize; they are only counted
                      // for blocks after the last real position
    }
}

// lb[c] = number of rows whose prefix code is < c.  Row r fills the codes
// (code(r-1), code(r)]; row 0 fills [0, code(0)]; the codes past the last
// row get Tsize.
__global__ void lb_build_kernel(const uint8_t *T, int64_t Tsize, const int64_t *SA, int64_t *lb) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r <= Tsize;
         r += (int64_t)gridDim.x * blockDim.x) {
        const int64_t cur = r < Tsize ? text_code(T, Tsize, SA[r]) : kCodes;
        const int64_t prev = r > 0 ? text_code(T, Tsize, SA[r - 1]) : -1;
        for (int64_t c = prev + 1; c <= cur && c <= kCodes; ++c) lb[c] = r;
    }
}

// --------------------------------------------------------------- seeding

// One thread per searched query position (query_find_suffixes,
// src/query.c:104-131).  Writes two cursor slots per position: slot 0 the
// bound row with direction +1, slot 1 the row before with direction -1
// (len < min_hit_length marks a slot that is not inserted).
__global__ void seed_kernel(DevIndex ix, SeedArgs a) {
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < a.npos;
         g += (int64_t)gridDim.x * blockDim.x) {
        // query of this position
        int lo = 0, hi = a.nq - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (a.pos_base[mid] <= g) lo = mid; else hi = mid - 1;
        }
        const int q = lo;
        const int i = (int)(g - a.pos_base[q]);
        const uint8_t *Q = a.qcat + a.qoff[q];
        const int qlen = a.qlen[q];
        Cursor c0, c1;
        c0.row = -1; c0.off = i; c0.dir = 1; c0.cpos = 0; c0.cn = a.chain; c0.prot = -1; c0.score = 0; c0.len = -1;
        c1.row = -1; c1.off = i; c1.dir = -1; c1.cpos = 0; c1.cn = a.chain; c1.prot = -1; c1.score = 0; c1.len = -1;
        if (Q[i] != 'V') {                     // _bad_prefix: internal 'V' = X
            const int64_t pos = lower_bound(ix, Q + i, qlen - i);
            if (a.lb_out) a.lb_out[g] = pos;
            if (pos >= ix.sa_rows) {
                atomicOr(&a.qstatus[q], TPZ_Q_SA_END);
            } else {
                int sc = 0;
                const int64_t t0 = ix.SA[pos];
                int ln = hsp_at(ix, t0, Q, qlen, i, a.sub, &sc);
                c0.row = pos; c0.score = sc; c0.len = ln;
                c0.prot = (int32_t)protein_of(ix, t0);
                if (pos != 0) {
                    sc = 0;
                    const int64_t t1 = ix.SA[pos - 1];
                    ln = hsp_at(ix, t1, Q, qlen, i, a.sub, &sc);
                    c1.row = pos - 1; c1.score = sc; c1.len = ln;
                    c1.prot = (int32_t)protein_of(ix, t1);
                }
            }
        } else if (a.lb_out) {
            a.lb_out[g] = -2;
        }
        a.cursors[2 * g] = c0;
        a.cursors[2 * g + 1] = c1;
    }
}

// Cursors that enter the queue (the chain kernel computes kChain elements
// for each): block sums, one atomic per block.
__global__ void count_queued_kernel(const Cursor *cursors, int64_t n, int min_hit_length,
                                    unsigned long long *count) {
    __shared__ unsigned int part;
    if (threadIdx.x == 0) part = 0;
    __syncthreads();
    unsigned int mine = 0;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
         c += (int64_t)gridDim.x * blockDim.x)
        mine += cursors[c].len >= min_hit_length;
    atomicAdd(&part, mine);
    __syncthreads();
    if (threadIdx.x == 0 && part) atomicAdd(count, (unsigned long long)part);
}

// One thread per pattern: the sa_search idx of a whole pattern.
__global__ void lower_bound_kernel(DevIndex ix, const uint8_t *pcat, const int64_t *poff,
                                   const int32_t *plen, int64_t n, int64_t *out) {
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n;
         g += (int64_t)gridDim.x * blockDim.x)
        out[g] = lower_bound(ix, pcat + poff[g], plen[g]);
}

// The per-call sa_search (src/search.c:237-362) in one thread, with all
// three of its outputs.  The lower bound and the match count have one answer
// each, whatever the search; `last_position` is the common prefix length of
// P with the last row the reference's binary search compares in its first
// loop (P's length once a row starting with P is found), so this search
// probes the rows in that same order: the window [lo, lo + size) with its
// probe at lo + half, both halves' known prefix lengths carried (a suffix
// between two rows shares at least the smaller of their common prefixes with
// P, so comparisons start past it).
__device__ int cmp_from(const DevIndex &ix, int64_t suf, const uint8_t *P, int64_t m,
                        int64_t *match) {
    int64_t i = suf + *match, j = *match;
    int r = 0;
    while (i < ix.Tsize && j < m && (r = (int)ix.T[i] - (int)P[j]) == 0) { ++i; ++j; }
    *match = j;
    return r == 0 ? -(j != m) : r;
}

__global__ void sa_search_call_kernel(DevIndex ix, const uint8_t *P, int64_t m, int64_t *out3) {
    int64_t lo = 0, size = ix.Tsize, half = size >> 1, lm = 0, rm = 0, match = 0;
    bool found = false;
    while (size > 0) {
        match = lm < rm ? lm : rm;
        const int r = cmp_from(ix, ix.SA[lo + half], P, m, &match);
        if (r < 0) {
            lo += half + 1;
            half -= (size & 1) ^ 1;
            lm = match;
        } else if (r > 0) {
            rm = match;
        } else {
            found = true;
            break;
        }
        size = half;
        half >>= 1;
    }
    int64_t first = lo, count = 0;
    if (found) {
        // rows starting with P form one run: its first row, then its end
        int64_t a = 0, b = ix.Tsize;
        while (a < b) {
            const int64_t mid = a + ((b - a) >> 1);
            int64_t k = 0;
            if (cmp_from(ix, ix.SA[mid], P, m, &k) < 0) a = mid + 1; else b = mid;
        }
        first = a;
        b = ix.Tsize;
        while (a < b) {
            const int64_t mid = a + ((b - a) >> 1);
            int64_t k = 0;
            if (cmp_from(ix, ix.SA[mid], P, m, &k) == 0) a = mid + 1; else b = mid;
        }
        count = a - first;
    }
    out3[0] = first;
    out3[1] = count;
    out3[2] = match;
}

// One thread per (row, query offset) for the stage entry point.
__global__ void hsp_batch_kernel(DevIndex ix, const uint8_t *qcat, const int64_t *qoff,
                                 const int32_t *qlen, const int32_t *query_of, const int32_t *off,
                                 const int64_t *row, int64_t n, const int8_t *sub, int32_t *score,
                                 int32_t *len) {
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n;
         g += (int64_t)gridDim.x * blockDim.x) {
        const int q = query_of[g];
        const int64_t r = row[g];
        int sc = 0, ln = -2;
        if (r >= 0 && r < ix.sa_rows) ln = hsp_at(ix, ix.SA[r], qcat + qoff[q], qlen[q], off[g], sub, &sc);
        score[g] = sc;
        len[g] = ln;
    }
}

// ------------------------------------------------------------------ walk

__device__ __forceinline__ uint32_t hash32(uint32_t x) {
    x ^= x >> 16; x *= 0x7feb352dU; x ^= x >> 15; x *= 0x846ca68bU; x ^= x >> 16;
    return x;
}

// highest set bit index <= from, or -1
__device__ __forceinline__ int bits_max_le(const uint64_t *bits, int from) {
    int w = from >> 6;
    uint64_t m = bits[w] & (((from & 63) == 63) ? ~0ull : ((2ull << (from & 63)) - 1));
    for (;;) {
        if (m) return (w << 6) + 63 - __clzll(m);
        if (--w < 0) return -1;
        m = bits[w];
    }
}

// lowest set bit index >= from, or -1
__device__ __forceinline__ int bits_min_ge(const uint64_t *bits, int from, int nwords) {
    int w = from >> 6;
    if (w >= nwords) return -1;
    uint64_t m = bits[w] & (~0ull << (from & 63));
    for (;;) {
        if (m) return (w << 6) + __ffsll(m) - 1;
        if (++w >= nwords) return -1;
        m = bits[w];
    }
}

// packed chain element: score in the low half, length in the high half
constexpr int kLenEnd = -1000;      // row outside [0, 8*Tsize): the cursor is freed
constexpr int kLenFault = -2000;    // row past the zero-filled SA page
__device__ __forceinline__ uint32_t pack_elem(int score, int len) {
    return (uint32_t)(uint16_t)(int16_t)score | ((uint32_t)(uint16_t)(int16_t)len << 16);
}
__device__ __forceinline__ int elem_score(uint32_t e) { return (int)(int16_t)(e & 0xFFFFu); }
__device__ __forceinline__ int elem_len(uint32_t e) { return (int)(int16_t)(e >> 16); }

// The chain element of a cursor `step` rows past `row` (step >= 1): the
// sa_hsp (src/suffix.c:47) of suffix_increment's next row, or a marker; and
// the protein of that row (db_index, the hitlist's key), -1 with a marker.
__device__ __forceinline__ uint32_t chain_elem(const DevIndex &ix, int64_t row, int dir, int step,
                                               const uint8_t *Q, int qlen, int off,
                                               const int8_t *sub, int32_t *prot) {
    const int64_t nr = row + (int64_t)dir * step;
    *prot = -1;
    if (nr < 0 || nr >= 8 * ix.Tsize) return pack_elem(0, kLenEnd);
    if (nr >= ix.sa_rows) return pack_elem(0, kLenFault);
    int sc = 0;
    const int64_t pos = ix.SA[nr];
    const int ln = hsp_at(ix, pos, Q, qlen, off, sub, &sc);
    *prot = (int32_t)protein_of(ix, pos);
    return pack_elem(sc, ln);
}

// One thread per (cursor, element): the first kChain chain elements of every
// queued cursor, so that the walk, whose pops run one after another, finds
// them ready.  Elements a cursor never reaches are computed and not used.
__global__ void chain_kernel(DevIndex ix, SeedArgs a, int min_hit_length, uint32_t *cache,
                             int32_t *cprot) {
    const int64_t total = 2 * a.npos * kChain;
    for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < total;
         x += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = x / kChain;
        const int e = (int)(x % kChain);
        const Cursor cu = a.cursors[c];
        if (cu.len < min_hit_length) continue;          // never queued
        const int64_t g = c >> 1;
        int lo = 0, hi = a.nq - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (a.pos_base[mid] <= g) lo = mid; else hi = mid - 1;
        }
        int32_t pr;
        cache[x] = chain_elem(ix, cu.row, cu.dir, e + 1, a.qcat + a.qoff[lo], a.qlen[lo], cu.off,
                              a.sub, &pr);
        cprot[x] = pr;
    }
}

struct HitView {
    int32_t *hprot, *hscore, *hlen, *hoff, *hprev, *hnext, *hfree;   // cap+1 slots
    int32_t *bhead, *btail;      // kSMax per-score lists (head = oldest)
    uint64_t *bbits;
    int32_t *hkey, *hval;        // protein -> slot, open addressing
};

__device__ __forceinline__ HitView hit_view(const WalkArgs &a, int q) {
    uint8_t *base = a.scratch + (size_t)q * a.scratch_per_query;
    HitView v;
    size_t o = 0;
    auto take = [&](size_t bytes) { uint8_t *p = base + o; o += (bytes + 15) & ~(size_t)15; return p; };
    const size_t ns = (size_t)a.max_cap + 1;
    v.hprot = (int32_t *)take(4 * ns);
    v.hscore = (int32_t *)take(4 * ns);
    v.hlen = (int32_t *)take(4 * ns);
    v.hoff = (int32_t *)take(4 * ns);
    v.hprev = (int32_t *)take(4 * ns);
    v.hnext = (int32_t *)take(4 * ns);
    v.hfree = (int32_t *)take(4 * ns);
    v.bhead = (int32_t *)take(4 * (size_t)kSMax);
    v.btail = (int32_t *)take(4 * (size_t)kSMax);
    v.bbits = (uint64_t *)take(8 * (size_t)(kSMax / 64));
    v.hkey = (int32_t *)take(4 * (size_t)a.hash_size);
    v.hval = (int32_t *)take(4 * (size_t)a.hash_size);
    return v;
}

// One warp per query.  Lane 0 runs the pop loop of
// query_fetch_alignment_batch (src/query.c:151-157) over pqueue_next
// (priority_queue.c:36-56) and hitlist_add (hit.c:126-193) exactly, with the
// per-score cursor stacks in shared memory.  A cursor's next chain elements
// (sa_hsp at rows row+dir, row+2dir, ...) come from a 32-entry per-cursor
// cache that all 32 lanes refill in one go whenever lane 0 pops a cursor
// whose cache is used up, so consecutive pops of a cursor cost no sa_hsp.
// Elements past the end of a chain are computed and never used.
__global__ void __launch_bounds__(kWalkWarps * 32) walk_kernel(DevIndex ix, WalkArgs a) {
    constexpr int NW = kSMax / 64;
    __shared__ int16_t s_qhead[kWalkWarps][kSMax];
    __shared__ uint64_t s_qbits[kWalkWarps][NW];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int q = blockIdx.x * kWalkWarps + wib;
    if (q >= a.nq) return;
    int16_t *qhead = s_qhead[wib];
    uint64_t *qbits = s_qbits[wib];
    const uint8_t *Q = a.qcat + a.qoff[q];
    const int qlen = a.qlen[q];
    const int minlen = a.min_hit_length;
    const int64_t cbase = a.cursor_base[q];
    const int ncur = (int)(a.cursor_base[q + 1] - cbase);
    Cursor *cur = a.cursors + cbase;
    int32_t *qnext = a.qnext + cbase;
    uint32_t *cache = a.ccache + cbase * kChain;
    int32_t *cprot = a.cprot + cbase * kChain;
    HitView v = hit_view(a, q);
    const int cap = qlen > 3000 ? (int)(1.5 * a.num_hits) : a.alignments;   // hit.c:106-109

    // ---- cooperative initialisation
    for (int i = lane; i < kSMax; i += 32) {
        qhead[i] = -1;
        v.bhead[i] = -1;
        v.btail[i] = -1;
    }
    for (int i = lane; i < NW; i += 32) { qbits[i] = 0; v.bbits[i] = 0; }
    for (int i = lane; i < a.hash_size; i += 32) v.hkey[i] = -1;
    for (int i = lane; i <= cap; i += 32) v.hfree[i] = cap - i;
    __syncwarp();

    int qmax = -1;
    int64_t qsize = 0;
    int nfree = cap + 1, hsize = 0, hmin = kSMax;
    const uint32_t hmask = (uint32_t)a.hash_size - 1;
    int64_t npops = 0, counter = 0, refills = 0;
    int status = 0;
    PopRec *trace = a.trace ? a.trace + (int64_t)q * a.trace_cap : nullptr;
    if (lane == 0) {
        // the queue in seeding insertion order
        for (int c = 0; c < ncur; ++c) {
            if (cur[c].len >= minlen) {
                const int sc = cur[c].score;
                qnext[c] = qhead[sc];
                qhead[sc] = (int16_t)c;
                qbits[sc >> 6] |= 1ull << (sc & 63);
                if (sc > qmax) qmax = sc;
                ++qsize;
            }
        }
    }

    for (;;) {
        // ---- lane 0: pop the newest cursor of the highest score
        int c = -1, need = 0, off = 0, dir = 0;
        int64_t row = 0;
        Cursor cc;
        if (lane == 0 && qsize > 0) {
            const int s = qmax;
            c = qhead[s];
            cc = cur[c];
            const int nx = qnext[c];
            qhead[s] = (int16_t)nx;
            if (nx < 0) {
                qbits[s >> 6] &= ~(1ull << (s & 63));
                qmax = s > 0 ? bits_max_le(qbits, s - 1) : -1;
            }
            --qsize;
            row = cc.row; off = cc.off; dir = cc.dir;
            need = cc.cpos >= cc.cn;
        }
        c = __shfl_sync(0xFFFFFFFFu, c, 0);
        if (c < 0) break;
        need = __shfl_sync(0xFFFFFFFFu, need, 0);
        uint32_t elem = 0;
        int32_t eprot = -1;
        if (need) {
            ++refills;
            // all lanes: the next 32 rows of this cursor
            row = __shfl_sync(0xFFFFFFFFu, row, 0);
            off = __shfl_sync(0xFFFFFFFFu, off, 0);
            dir = __shfl_sync(0xFFFFFFFFu, dir, 0);
            elem = chain_elem(ix, row, dir, lane + 1, Q, qlen, off, a.sub, &eprot);
            cache[(int64_t)c * kChain + lane] = elem;
            cprot[(int64_t)c * kChain + lane] = eprot;
            __syncwarp();
        }
        int stop = 0;
        if (lane == 0) {
            if (need) {
                cc.cpos = 1;
                cc.cn = 32;
            } else {
                elem = cache[(int64_t)c * kChain + cc.cpos];
                eprot = cprot[(int64_t)c * kChain + cc.cpos];
                cc.cpos++;
            }
            const int gs = cc.score, gl = cc.len, gprot = cc.prot;
            // suffix_increment + suffix_active
            const int ln = elem_len(elem);
            if (ln == kLenFault) {
                status |= TPZ_Q_SA_END;
                stop = 1;
            } else {
                if (ln != kLenEnd) {
                    cc.row = row + dir;
                    cc.len = ln;
                    cc.prot = eprot;
                    if (ln >= minlen) {
                        const int sc = elem_score(elem);
                        cc.score = sc;
                        qnext[c] = qhead[sc];
                        qhead[sc] = (int16_t)c;
                        qbits[sc >> 6] |= 1ull << (sc & 63);
                        if (sc > qmax) qmax = sc;
                        ++qsize;
                    }
                }
                cur[c] = cc;

                // ---- hitlist_add (every queued row is below sa_rows: seeding and
                // the advance above stop at the first row past it)
                bool counted = false;
                if (hsize >= cap && hmin >= gs) {
                    counted = true;            // full and the worst hit is at least as good
                } else {
                    const int p = gprot;      // protein_of(ix, ix.SA[row])
                    uint32_t hh = hash32((uint32_t)p) & hmask;
                    while (v.hkey[hh] != -1 && v.hkey[hh] != p) hh = (hh + 1) & hmask;
                    if (v.hkey[hh] == -1) {
                        // new protein: newest entry of its score list
                        const int slot = v.hfree[--nfree];
                        v.hprot[slot] = p; v.hscore[slot] = gs; v.hlen[slot] = gl; v.hoff[slot] = off;
                        v.hnext[slot] = -1;
                        v.hprev[slot] = v.btail[gs];
                        if (v.btail[gs] >= 0) v.hnext[v.btail[gs]] = slot; else v.bhead[gs] = slot;
                        v.btail[gs] = slot;
                        v.bbits[gs >> 6] |= 1ull << (gs & 63);
                        if (gs < hmin) hmin = gs;
                        v.hkey[hh] = p; v.hval[hh] = slot;
                        ++hsize;
                        if (hsize > cap) {
                            // evict the oldest entry of the smallest score
                            const int m = hmin;
                            const int w = v.bhead[m];
                            v.bhead[m] = v.hnext[w];
                            if (v.bhead[m] >= 0) v.hprev[v.bhead[m]] = -1; else {
                                v.btail[m] = -1;
                                v.bbits[m >> 6] &= ~(1ull << (m & 63));
                                const int nm = bits_min_ge(v.bbits, m + 1, NW);
                                hmin = nm < 0 ? kSMax : nm;
                            }
                            // delete its protein from the table (backward shift)
                            const int wp = v.hprot[w];
                            uint32_t i = hash32((uint32_t)wp) & hmask;
                            while (v.hkey[i] != wp) i = (i + 1) & hmask;
                            uint32_t j = i;
                            for (;;) {
                                j = (j + 1) & hmask;
                                if (v.hkey[j] == -1) break;
                                const uint32_t k = hash32((uint32_t)v.hkey[j]) & hmask;
                                // move j into the hole at i when its home k is not in (i, j]
                                const bool keep = (i <= j) ? (i < k && k <= j) : (i < k || k <= j);
                                if (!keep) {
                                    v.hkey[i] = v.hkey[j]; v.hval[i] = v.hval[j];
                                    i = j;
                                }
                            }
                            v.hkey[i] = -1;
                            v.hfree[nfree++] = w;
                            --hsize;
                        }
                        counted = true;
                    } else {
                        const int h = v.hval[hh];
                        const int os = v.hscore[h];
                        if (os < gs) {
                            // rb_reput: unlink, re-key, append as newest
                            if (v.hprev[h] >= 0) v.hnext[v.hprev[h]] = v.hnext[h]; else v.bhead[os] = v.hnext[h];
                            if (v.hnext[h] >= 0) v.hprev[v.hnext[h]] = v.hprev[h]; else v.btail[os] = v.hprev[h];
                            if (v.bhead[os] < 0) {
                                v.bbits[os >> 6] &= ~(1ull << (os & 63));
                                if (hmin == os) {
                                    const int nm = bits_min_ge(v.bbits, os + 1, NW);
                                    hmin = nm < 0 ? kSMax : nm;
                                }
                            }
                            v.hscore[h] = gs; v.hlen[h] = gl;
                            v.hnext[h] = -1;
                            v.hprev[h] = v.btail[gs];
                            if (v.btail[gs] >= 0) v.hnext[v.btail[gs]] = h; else v.bhead[gs] = h;
                            v.btail[gs] = h;
                            v.bbits[gs >> 6] |= 1ull << (gs & 63);
                            if (gs < hmin) hmin = gs;
                        }
                    }
                }
                if (trace && npops < a.trace_cap) {
                    PopRec r; r.row = row; r.off = off; r.score = gs; r.len = gl; r.counted = counted;
                    trace[npops] = r;
                }
                ++npops;
                if (counted && ++counter == a.seeds) stop = 1;
            }
        }
        stop = __shfl_sync(0xFFFFFFFFu, stop, 0);
        if (stop) break;
    }

    if (lane == 0) {
        // ---- hitlist in traversal order: score descending, newest first
        Hit *out = a.hits + (int64_t)q * a.max_cap;
        int n = 0;
        for (int sc = bits_max_le(v.bbits, kSMax - 1); sc >= 0;
             sc = sc > 0 ? bits_max_le(v.bbits, sc - 1) : -1) {
            for (int h = v.btail[sc]; h >= 0; h = v.hprev[h]) {
                Hit o;
                o.protein = v.hprot[h]; o.gapless_score = v.hscore[h]; o.gapless_length = v.hlen[h];
                o.suffix_offset = v.hoff[h];
                out[n++] = o;
            }
        }
        QueryOut qo;
        qo.nhits = n; qo.npops = npops; qo.ncounted = counter; qo.status = status | a.qstatus[q];
        qo.refills = refills;
        a.qout[q] = qo;
    }
}

}  // namespace search
}  // namespace tpz
