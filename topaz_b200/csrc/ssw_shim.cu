// ssw_shim.cu -- per-call SSW entry points (include/topaz_b200_ssw.h) over
// the device Smith-Waterman and the host statistics.
#include <stdlib.h>
#include <string.h>

#include <algorithm>

#include "../../include/topaz_b200_ssw.h"
extern "C" {
#include "../host/tpzh.h"
}
#include "search_internal.cuh"

// the library-owned part of a profile: the matrix and the device copy of
// the query
struct tpz_ssw_device {
    int8_t *d_read;
    int8_t mat[625];
};

namespace {

// per host thread: device copies of the subject and the result of one call
struct ShimBufs {
    int8_t *ref = nullptr;
    int64_t cap = 0;
    int32_t *meta = nullptr;    // qlen, slen, score, ref_end, read_end, status
    int64_t *offs = nullptr;    // qoff, soff (both 0)
    ~ShimBufs() {
        if (ref) cudaFree(ref);
        if (meta) cudaFree(meta);
        if (offs) cudaFree(offs);
    }
};

int shim_bufs(ShimBufs **out, int64_t refLen) {
    static thread_local ShimBufs b;
    if (!b.meta) {
        TPZ_CUDA(cudaMalloc((void **)&b.meta, 8 * sizeof(int32_t)));
        TPZ_CUDA(cudaMalloc((void **)&b.offs, 2 * sizeof(int64_t)));
        TPZ_CUDA(cudaMemset(b.offs, 0, 2 * sizeof(int64_t)));
    }
    if (refLen + 1 > b.cap) {
        if (b.ref) cudaFree(b.ref);
        b.ref = nullptr;
        b.cap = std::max<int64_t>(refLen + 1, 4096);
        TPZ_CUDA(cudaMalloc((void **)&b.ref, b.cap));
    }
    *out = &b;
    return TPZ_OK;
}

}  // namespace

extern "C" {

s_profile *ssw_init(const int8_t *read, const int32_t readLen, const int8_t *mat, const int32_t n,
                    const int8_t score_size) {
    if (!read || !mat || readLen < 1 || readLen > TPZ_SW_MAX_QLEN || n != 25 || score_size != 2) {
        tpz::set_error("ssw_init: need a read of 1..8192 residues, n = 25 and score_size = 2");
        return nullptr;
    }
    s_profile *p = (s_profile *)calloc(1, sizeof(s_profile));
    tpz_ssw_device *d = (tpz_ssw_device *)calloc(1, sizeof(tpz_ssw_device));
    if (!p || !d) { free(p); free(d); return nullptr; }
    p->read = (int8_t *)read;
    p->readLen = readLen;
    p->n = n;
    memcpy(d->mat, mat, 625);
    int mn = 0;
    for (int i = 0; i < 625; ++i) mn = std::min<int>(mn, mat[i]);
    p->bias = (uint8_t)(-mn);
    p->mat = d->mat;
    p->device = d;
    if (cudaMalloc((void **)&d->d_read, readLen) != cudaSuccess ||
        cudaMemcpy(d->d_read, read, readLen, cudaMemcpyHostToDevice) != cudaSuccess) {
        tpz::cuda_fail(cudaGetLastError(), "ssw_init");
        if (d->d_read) cudaFree(d->d_read);
        free(d);
        free(p);
        return nullptr;
    }
    return p;
}

void init_destroy(s_profile *p) {
    if (!p) return;
    if (p->device) {
        if (p->device->d_read) cudaFree(p->device->d_read);
        free(p->device);
    }
    free(p);
}

void init_destroy2(s_profile *p) {
    if (!p) return;
    free(p->read);
    init_destroy(p);
}

s_align *ssw_align(const s_profile *prof, const int8_t *ref, int32_t refLen,
                   const uint8_t weight_gapO, const uint8_t weight_gapE, const uint8_t flag,
                   const uint16_t filters, const int32_t filterd, const int32_t maskLen) {
    (void)flag; (void)filters; (void)filterd; (void)maskLen;
    if (!prof || !ref || refLen < 0) {
        tpz::set_error("ssw_align: bad arguments");
        return nullptr;
    }
    ShimBufs *b = nullptr;
    if (shim_bufs(&b, refLen)) return nullptr;
    cudaStream_t st = cudaStreamPerThread;
    int32_t h[8] = {prof->readLen, refLen, 0, 0, 0, -1, 0, 0};
    if (cudaMemcpyAsync(b->ref, ref, std::max<int32_t>(refLen, 1), cudaMemcpyHostToDevice, st) ||
        cudaMemcpyAsync(b->meta, h, sizeof h, cudaMemcpyHostToDevice, st)) {
        tpz::cuda_fail(cudaGetLastError(), "ssw_align");
        return nullptr;
    }
    int rc;
    if (prof->readLen <= 1024) {
        rc = tpz_sw_align_one(prof->device->d_read, prof->readLen, b->ref, refLen,
                              prof->device->mat, weight_gapO, weight_gapE, b->meta + 2, st);
    } else {
        rc = tpz::sw::batch_device_x(1, prof->device->d_read, b->offs, b->meta, b->ref, b->offs + 1,
                                     b->meta + 1, prof->device->mat, weight_gapO, weight_gapE,
                                     b->meta + 2, b->meta + 3, b->meta + 4, b->meta + 5, st,
                                     nullptr, nullptr, 0);
    }
    if (rc) return nullptr;
    if (cudaMemcpyAsync(h, b->meta, sizeof h, cudaMemcpyDeviceToHost, st) ||
        cudaStreamSynchronize(st)) {
        tpz::cuda_fail(cudaGetLastError(), "ssw_align");
        return nullptr;
    }
    if (h[5] != TPZ_SW_OK) return nullptr;          // dropped at 32767, as ssw_align
    s_align *r = (s_align *)calloc(1, sizeof(s_align));
    if (!r) return nullptr;
    r->score1 = (uint16_t)h[2];
    r->score2 = 0;
    r->ref_begin1 = -1;
    r->ref_end1 = h[3];
    r->read_begin1 = -1;
    r->read_end1 = h[4];
    r->ref_end2 = -1;
    r->cigar = nullptr;
    r->cigarLen = 0;
    return r;
}

void align_destroy(s_align *a) { free(a); }

int ssw_align_stats(const s_profile *prof, const int8_t *ref, int32_t refLen,
                    const uint8_t weight_gapO, const uint8_t weight_gapE, const int32_t maskLen,
                    int32_t read_end1, int32_t ref_end1, uint16_t score1, int32_t *read_begin1,
                    int32_t *ref_begin1, int32_t *length, int32_t *gapopen, int32_t *mismatch,
                    double *identity) {
    (void)maskLen;
    tpzh_stats s;
    const int rc = tpzh_align_stats(prof->read, prof->readLen, ref, refLen, prof->device->mat, weight_gapO,
                                    weight_gapE, read_end1, ref_end1, score1, &s);
    *read_begin1 = s.qstart;
    *ref_begin1 = s.sstart;
    *length = s.length;
    *gapopen = s.gapopen;
    *mismatch = s.mismatch;
    *identity = s.identity;
    return rc;
}

}  // extern "C"
