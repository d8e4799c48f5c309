// tpz_common.cu -- error reporting, matrix tables, device queries.
#include <stdio.h>
#include <string.h>

#include <mutex>
#include <string>
#include <vector>

#include "tpz_common.cuh"
#include "tpz_matrices.inc"

namespace tpz {

static thread_local std::string g_last_error;

void set_error(const std::string &msg) { g_last_error = msg; }

int cuda_fail(cudaError_t e, const char *what) {
    char buf[512];
    snprintf(buf, sizeof buf, "CUDA error %d (%s) in %s", (int)e, cudaGetErrorString(e), what);
    set_error(buf);
    return e == cudaErrorMemoryAllocation ? TPZ_E_NOMEM : TPZ_E_CUDA;
}

// The order of rows and columns in every table text.
static const char kMatrixOrder[] = "ARNDCQEGHILKMFPSTWYVBJZX*";

static int parse_matrix(const char *text, int8_t *out) {
    // line 0: column letters; lines 1..25: row letter then 25 integers
    const char *p = strchr(text, '\n');
    if (!p) return -1;
    ++p;
    for (int r = 0; r < 25; ++r) {
        while (*p == ' ') ++p;
        if (*p != kMatrixOrder[r]) return -1;
        ++p;
        for (int c = 0; c < 25; ++c) {
            char *end;
            long v = strtol(p, &end, 10);
            if (end == p) return -1;
            out[r * 25 + c] = (int8_t)v;
            p = end;
        }
        p = strchr(p, '\n');
        if (!p) return -1;
        ++p;
    }
    return 0;
}

int matrix_by_name(const char *name, int8_t *out625) {
    if (!name || !out625) {
        set_error("tpz_matrix: NULL argument");
        return TPZ_E_ARG;
    }
    for (int i = 0; i < TPZ_NUM_MATRICES; ++i) {
        if (strcmp(name, TPZ_MATRIX_NAMES[i]) == 0) {
            if (parse_matrix(TPZ_MATRIX_TEXTS[i], out625) != 0) {
                set_error("internal: matrix table text is malformed");
                return TPZ_E_ARG;
            }
            return TPZ_OK;
        }
    }
    set_error(std::string("unknown substitution matrix \"") + name + "\"");
    return TPZ_E_ARG;
}

void keep_pool_memory() {
    static thread_local int done_dev = -1;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev == done_dev) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    done_dev = dev;
}

int sm_count() {
    static std::mutex mu;
    static std::vector<int> cache;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 148;
    std::lock_guard<std::mutex> lk(mu);
    if ((int)cache.size() <= dev) cache.resize(dev + 1, 0);
    if (!cache[dev]) {
        int n = 0;
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        cache[dev] = n > 0 ? n : 148;
    }
    return cache[dev];
}

}  // namespace tpz

extern "C" {

const char *tpz_last_error(void) { return tpz::g_last_error.c_str(); }

const char *tpz_version(void) { return "topaz_b200 0.1 (sm_100a)"; }

int tpz_matrix(const char *name, int8_t *out625) { return tpz::matrix_by_name(name, out625); }

}  // extern "C"
