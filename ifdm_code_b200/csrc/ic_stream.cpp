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

static std::string upload_chunk(const IcChunk &ch, bool ref1, float *d_pos, float *d_vel, int device,
                                size_t piece) {
    cudaError_t ce = cudaSetDevice(device);
    if (ce != cudaSuccess) return cudaGetErrorString(ce);
    cudaStream_t st = nullptr;
    char *buf[2] = {nullptr, nullptr};
    cudaEvent_t ev[2] = {nullptr, nullptr};
    bool used[2] = {false, false};
    std::string err;
    const int fd = open(ch.path.c_str(), O_RDONLY);
    auto cuda_ok = [&](cudaError_t e, const char *what) {
        if (e != cudaSuccess && err.empty()) err = std::string(what) + ": " + cudaGetErrorString(e);
        return e == cudaSuccess;
    };
    if (fd < 0) err = " cannot read IC file !! " + ch.path;
    if (err.empty() && cuda_ok(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate")) {
        for (int k = 0; k < 2 && err.empty(); ++k) {
            cuda_ok(cudaHostAlloc(reinterpret_cast<void **>(&buf[k]), piece, cudaHostAllocDefault), "cudaHostAlloc");
            if (err.empty()) cuda_ok(cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming), "cudaEventCreate");
        }
    }
    int turn = 0;
    // one block of the file -> device, through the two pinned buffers
    auto stream_block = [&](long file_off, size_t nbytes, char *dst) {
        for (size_t off = 0; off < nbytes && err.empty(); off += piece) {
            const int k = turn++ & 1;
            const size_t len = std::min(piece, nbytes - off);
            if (used[k] && !cuda_ok(cudaEventSynchronize(ev[k]), "cudaEventSynchronize")) return;
            if (!pread_all(fd, buf[k], len, off_t(file_off + off))) {
                err = "truncated Gadget blocks " + ch.path;
                return;
            }
            if (!cuda_ok(cudaMemcpyAsync(dst + off, buf[k], len, cudaMemcpyHostToDevice, st), "cudaMemcpyAsync")) return;
            cuda_ok(cudaEventRecord(ev[k], st), "cudaEventRecord");
            used[k] = true;
        }
    };
    const long body = ch.base + (ref1 ? ch.lg : 0);
    if (err.empty()) stream_block(pos_offset(), size_t(12 * ch.n), reinterpret_cast<char *>(d_pos + 3 * body));
    if (err.empty()) stream_block(vel_offset(ch.n), size_t(12 * ch.n), reinterpret_cast<char *>(d_vel + 3 * body));
    if (err.empty() && ref1) {
        const size_t gb = size_t(12 * ch.lg);
        const long tail = body + ch.n - ch.lg;
        if (gb) {
            cuda_ok(cudaMemcpyAsync(d_pos + 3 * ch.base, d_pos + 3 * tail, gb, cudaMemcpyDeviceToDevice, st), "ghosts");
            cuda_ok(cudaMemcpyAsync(d_vel + 3 * ch.base, d_vel + 3 * tail, gb, cudaMemcpyDeviceToDevice, st), "ghosts");
        }
        cuda_ok(cudaMemsetAsync(d_pos + 3 * (body + ch.n), 0, 12, st), "cudaMemsetAsync");
        cuda_ok(cudaMemsetAsync(d_vel + 3 * (body + ch.n), 0, 12, st), "cudaMemsetAsync");
    }
    if (st) cuda_ok(cudaStreamSynchronize(st), "cudaStreamSynchronize");
    for (int k = 0; k < 2; ++k) {
        if (buf[k]) cudaFreeHost(buf[k]);
        if (ev[k]) cudaEventDestroy(ev[k]);
    }
    if (st) cudaStreamDestroy(st);
    if (fd >= 0) close(fd);
    return err;
}

std::string ic_upload(const std::vector<IcChunk> &chunks, bool ref1, float *d_pos, float *d_vel, int device,
                      size_t piece_bytes) {
    std::vector<std::string> errs(chunks.size());
    std::vector<std::thread> pool;
    for (size_t c = 0; c < chunks.size(); ++c)
        pool.emplace_back([&, c] { errs[c] = upload_chunk(chunks[c], ref1, d_pos, d_vel, device, piece_bytes); });
    for (auto &t : pool) t.join();
    for (auto &e : errs)
        if (!e.empty()) return e;
    return "";
}

}  // namespace ifdm
