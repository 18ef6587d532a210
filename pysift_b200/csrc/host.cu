// Host-side helpers of the drop-in surface (no kernels).
//
//   pysift_host_copy   memcpy split over a small persistent pool of host
//                      threads: the staging copy of a host image into
//                      page-locked memory before its upload (a single
//                      thread copies about 18 GB/s, so one 1280x960 BGR
//                      view costs 0.2 ms before its host-to-device copy can
//                      start).
#include <unistd.h>

#include <algorithm>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "common.cuh"

namespace pysift {
namespace {

// Workers sleep on a condition variable between jobs; a job is one buffer
// cut into `parts` pieces, piece 0 copied by the calling thread and piece
// i > 0 by worker i - 1.  One job at a time (callers serialise on `call`).
struct CopyPool {
    std::mutex call;
    std::mutex m;
    std::condition_variable go, done;
    uint64_t gen = 0;
    int pending = 0;
    int parts = 0;
    char* dst = nullptr;
    const char* src = nullptr;
    size_t bytes = 0, piece = 0;
    int n_workers = 0;
    pid_t owner = 0;

    explicit CopyPool(int workers) : n_workers(workers), owner(getpid()) {
        for (int i = 0; i < workers; ++i) std::thread([this, i] { run(i + 1); }).detach();
    }
    void copy_piece(int p) const {
        const size_t lo = (size_t)p * piece;
        if (lo >= bytes) return;
        std::memcpy(dst + lo, src + lo, std::min(piece, bytes - lo));
    }
    void run(int p) {
        uint64_t seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(m);
                go.wait(lk, [&] { return gen != seen; });
                seen = gen;
                if (p >= parts) continue;
            }
            copy_piece(p);
            std::lock_guard<std::mutex> lk(m);
            if (--pending == 0) done.notify_one();
        }
    }
    void copy(void* d, const void* s, size_t n, int want) {
        std::lock_guard<std::mutex> serial(call);
        const int k = std::max(1, std::min(want, n_workers + 1));
        {
            std::lock_guard<std::mutex> lk(m);
            dst = static_cast<char*>(d);
            src = static_cast<const char*>(s);
            bytes = n;
            parts = k;
            piece = ((n + k - 1) / k + 4095) & ~(size_t)4095;  // whole pages per piece
            pending = k - 1;
            ++gen;
        }
        go.notify_all();
        copy_piece(0);
        std::unique_lock<std::mutex> lk(m);
        done.wait(lk, [&] { return pending == 0; });
    }
};

CopyPool* g_pool = nullptr;
std::mutex g_pool_m;

// The pool of this process (a child after fork() has none of its parent's
// threads, so it builds its own; the parent's object is left alone).
CopyPool* copy_pool() {
    std::lock_guard<std::mutex> lk(g_pool_m);
    if (!g_pool || g_pool->owner != getpid()) {
        const unsigned hw = std::thread::hardware_concurrency();
        const int workers = std::max(0, std::min(7, (int)(hw ? hw : 1) - 1));
        g_pool = new CopyPool(workers);  // lives until exit; its workers are detached
    }
    return g_pool;
}

}  // namespace
}  // namespace pysift

extern "C" {

int pysift_host_copy(void* dst, const void* src, size_t bytes, int32_t n_threads) {
    PYSIFT_CHECK_ARG(bytes == 0 || (dst && src), "NULL pointer argument");
    PYSIFT_CHECK_ARG(n_threads >= 1 && n_threads <= 64, "n_threads must be 1..64");
    if (bytes == 0) return PYSIFT_OK;
    // below 1 MiB a single memcpy is as fast as waking the workers
    if (n_threads == 1 || bytes < ((size_t)1 << 20)) {
        std::memcpy(dst, src, bytes);
        return PYSIFT_OK;
    }
    pysift::copy_pool()->copy(dst, src, bytes, n_threads);
    return PYSIFT_OK;
}

}  // extern "C"
