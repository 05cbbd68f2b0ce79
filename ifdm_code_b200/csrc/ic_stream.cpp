// ic_stream.cpp -- see ic_stream.hpp.
#include "ic_stream.hpp"

#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <thread>

namespace ifdm {

namespace {

// Gadget-1 block offsets of one chunk file: int 256, header, int 256, then
// int, pos f32[3n], int, int, vel f32[3n], int (src/gadget_IC.h:279-300)
constexpr long kHeadBytes = 4 + 256 + 4;
long pos_offset() { return kHeadBytes + 4; }
long vel_offset(long n) { return kHeadBytes + 4 + 12 * n + 4 + 4; }

bool pread_all(int fd, void *dst, size_t n, off_t off) {
    char *p = static_cast<char *>(dst);
    while (n > 0) {
        const ssize_t r = pread(fd, p, n, off);
        if (r < 0 && errno == EINTR) continue;
        if (r <= 0) return false;
        p += r;
        n -= size_t(r);
        off += r;
    }
    return true;
}

// trailing particles with x beyond the last cell centre (pn > 0), read
// backwards through the position block in pieces
bool count_ghosts(int fd, long n, double xg_last, long *lg) {
    constexpr long P = 1 << 16;
    std::vector<float> buf(3 * P);
    long count = 0, hi = n;  // particles [lo, hi) in buf
    while (hi > 1) {
        const long lo = std::max(1L, hi - P);
        if (!pread_all(fd, buf.data(), size_t(12 * (hi - lo)), off_t(pos_offset() + 12 * lo))) return false;
        for (long pn = hi - 1; pn >= lo; --pn) {
            if (xg_last < buf[3 * (pn - lo)]) ++count;
            else {
                *lg = count;
                return true;
            }
        }
        hi = lo;
    }
    *lg = count;
    return true;
}

}  // namespace

std::string ic_scan_chunks(const std::string &icpath, int nchunks, int N, bool ref1, std::vector<IcChunk> *out,
                           long *np_total) {
    out->clear();
    long slots = 0;
    for (int c = 0; c < nchunks; ++c) {
        IcChunk ch;
        ch.path = icpath + "." + std::to_string(c);
        const int fd = open(ch.path.c_str(), O_RDONLY);
        if (fd < 0) return " cannot read IC file !! " + ch.path;
        std::string err;
        int b0 = 0;
        if (!pread_all(fd, &b0, 4, 0) || !pread_all(fd, &ch.h, sizeof(GadgetHeader), 4)) {
            err = "truncated Gadget header " + ch.path;
        } else {
            ch.n = ch.h.npart[1];
            struct stat st{};
            if (ch.n < 0) err = "bad particle count in " + ch.path;
            else if (fstat(fd, &st) != 0 || st.st_size < vel_offset(ch.n) + 12 * ch.n)
                err = "truncated Gadget blocks " + ch.path;
            else if (ref1) {
                const double Lg = ch.h.BoxSize / N;
                const double xg_last = (N - 1) * Lg + 0.5 * Lg;
                if (!count_ghosts(fd, ch.n, xg_last, &ch.lg)) err = "truncated Gadget blocks " + ch.path;
            }
        }
        close(fd);
        if (!err.empty()) return err;
        ch.base = slots;
        slots += ref1 ? ch.lg + ch.n + 1 : ch.n;
        out->push_back(ch);
    }
    *np_total = slots;
    return "";
}

namespace {

// a contiguous byte range of one chunk's position or velocity block and its
// place in the device arrays
struct Range {
    int chunk;
    long file_off;
    size_t bytes;
    char *dst;
};

}  // namespace

// worker w of W: the ranges w, w + W, ... through its own stream and two
// pinned buffers (one piece read while the previous one is copied)
static std::string upload_ranges(const std::vector<IcChunk> &chunks, const std::vector<Range> &ranges, int w,
                                 int W, int device, size_t piece) {
    cudaError_t ce = cudaSetDevice(device);
    if (ce != cudaSuccess) return cudaGetErrorString(ce);
    cudaStream_t st = nullptr;
    char *buf[2] = {nullptr, nullptr};
    cudaEvent_t ev[2] = {nullptr, nullptr};
    bool used[2] = {false, false};
    std::vector<int> fds(chunks.size(), -1);
    std::string err;
    auto cuda_ok = [&](cudaError_t e, const char *what) {
        if (e != cudaSuccess && err.empty()) err = std::string(what) + ": " + cudaGetErrorString(e);
        return e == cudaSuccess;
    };
    if (cuda_ok(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate")) {
        for (int k = 0; k < 2 && err.empty(); ++k) {
            cuda_ok(cudaHostAlloc(reinterpret_cast<void **>(&buf[k]), piece, cudaHostAllocDefault), "cudaHostAlloc");
            if (err.empty()) cuda_ok(cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming), "cudaEventCreate");
        }
    }
    int turn = 0;
    for (size_t r = size_t(w); r < ranges.size() && err.empty(); r += size_t(W)) {
        const Range &rg = ranges[r];
        const IcChunk &ch = chunks[size_t(rg.chunk)];
        if (fds[size_t(rg.chunk)] < 0) fds[size_t(rg.chunk)] = open(ch.path.c_str(), O_RDONLY);
        const int fd = fds[size_t(rg.chunk)];
        if (fd < 0) {
            err = " cannot read IC file !! " + ch.path;
            break;
        }
        for (size_t off = 0; off < rg.bytes && err.empty(); off += piece) {
            const int k = turn++ & 1;
            const size_t len = std::min(piece, rg.bytes - off);
            if (used[k] && !cuda_ok(cudaEventSynchronize(ev[k]), "cudaEventSynchronize")) break;
            if (!pread_all(fd, buf[k], len, off_t(rg.file_off + long(off)))) {
                err = "truncated Gadget blocks " + ch.path;
                break;
            }
            if (!cuda_ok(cudaMemcpyAsync(rg.dst + off, buf[k], len, cudaMemcpyHostToDevice, st), "cudaMemcpyAsync"))
                break;
            cuda_ok(cudaEventRecord(ev[k], st), "cudaEventRecord");
            used[k] = true;
        }
    }
    if (st) cuda_ok(cudaStreamSynchronize(st), "cudaStreamSynchronize");
    for (int k = 0; k < 2; ++k) {
        if (buf[k]) cudaFreeHost(buf[k]);
        if (ev[k]) cudaEventDestroy(ev[k]);
    }
    if (st) cudaStreamDestroy(st);
    for (int fd : fds)
        if (fd >= 0) close(fd);
    return err;
}

std::string ic_upload(const std::vector<IcChunk> &chunks, bool ref1, float *d_pos, float *d_vel, int device,
                      size_t piece_bytes) {
    // every block cut into ranges of a few pieces, spread over the workers
    const size_t span = 4 * piece_bytes;
    std::vector<Range> ranges;
    for (size_t c = 0; c < chunks.size(); ++c) {
        const IcChunk &ch = chunks[c];
        const long body = ch.base + (ref1 ? ch.lg : 0);
        const size_t bytes = size_t(12 * ch.n);
        char *dpos = reinterpret_cast<char *>(d_pos + 3 * body), *dvel = reinterpret_cast<char *>(d_vel + 3 * body);
        for (size_t off = 0; off < bytes; off += span) {
            const size_t len = std::min(span, bytes - off);
            ranges.push_back({int(c), pos_offset() + long(off), len, dpos + off});
            ranges.push_back({int(c), vel_offset(ch.n) + long(off), len, dvel + off});
        }
    }
    const int hw = int(std::thread::hardware_concurrency());
    const int W = int(std::max<size_t>(1, std::min<size_t>(ranges.size(), size_t(std::min(16, std::max(1, hw))))));
    std::vector<std::string> errs(static_cast<size_t>(W));
    std::vector<std::thread> pool;
    for (int w = 0; w < W; ++w)
        pool.emplace_back([&, w] { errs[size_t(w)] = upload_ranges(chunks, ranges, w, W, device, piece_bytes); });
    for (auto &t : pool) t.join();
    for (auto &e : errs)
        if (!e.empty()) return e;
    if (!ref1) return "";
    // ghosts (a device copy of each chunk's tail, in front of it) and the zero particle after it
    cudaStream_t st = nullptr;
    cudaError_t ce = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    for (size_t c = 0; c < chunks.size() && ce == cudaSuccess; ++c) {
        const IcChunk &ch = chunks[c];
        const long body = ch.base + ch.lg, tail = body + ch.n - ch.lg;
        const size_t gb = size_t(12 * ch.lg);
        if (gb) {
            ce = cudaMemcpyAsync(d_pos + 3 * ch.base, d_pos + 3 * tail, gb, cudaMemcpyDeviceToDevice, st);
            if (ce == cudaSuccess)
                ce = cudaMemcpyAsync(d_vel + 3 * ch.base, d_vel + 3 * tail, gb, cudaMemcpyDeviceToDevice, st);
        }
        if (ce == cudaSuccess) ce = cudaMemsetAsync(d_pos + 3 * (body + ch.n), 0, 12, st);
        if (ce == cudaSuccess) ce = cudaMemsetAsync(d_vel + 3 * (body + ch.n), 0, 12, st);
    }
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    if (st) cudaStreamDestroy(st);
    return ce == cudaSuccess ? "" : std::string("IC ghost copies: ") + cudaGetErrorString(ce);
}

}  // namespace ifdm
