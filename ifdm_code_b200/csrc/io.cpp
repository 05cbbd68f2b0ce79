// io.cpp -- snapshot, voutput and Gadget chunk I/O (formats in io.hpp).
#include "io.hpp"

#include <cstdio>
#include <cstring>

namespace ifdm {

std::string snapshot_path(const std::string &prefix, int t) { return prefix + "output" + std::to_string(t) + ".dat"; }

std::string write_snapshot(const std::string &path, double mfdm, double g_cm3, double a, const std::vector<double> &x,
                           const double *psi, size_t n3) {
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) return "cannot open " + path + " for writing";
    bool ok = std::fwrite(&mfdm, sizeof(double), 1, f) == 1;
    ok = ok && std::fwrite(&g_cm3, sizeof(double), 1, f) == 1;
    ok = ok && std::fwrite(&a, sizeof(double), 1, f) == 1;
    ok = ok && std::fwrite(x.data(), sizeof(double), x.size(), f) == x.size();
    ok = ok && std::fwrite(psi, 2 * sizeof(double), n3, f) == n3;
    ok = (std::fclose(f) == 0) && ok;
    return ok ? "" : "short write to " + path;
}

std::string read_snapshot(const std::string &path, int N, double *a, std::vector<double> *x, double *psi) {
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) return "ERROR: cannot find icpath  !!! " + path;
    double hdr[3];
    std::vector<double> xs(N);
    bool ok = std::fread(hdr, sizeof(double), 3, f) == 3;
    ok = ok && std::fread(xs.data(), sizeof(double), N, f) == size_t(N);
    if (ok && psi) {
        const size_t n3 = size_t(N) * N * N;
        ok = std::fseek(f, long((N + 3) * sizeof(double)), SEEK_SET) == 0;
        ok = ok && std::fread(psi, 2 * sizeof(double), n3, f) == n3;
    }
    std::fclose(f);
    if (!ok) return "truncated snapshot " + path;
    *a = hdr[2];
    if (x) *x = xs;
    return "";
}

std::string write_voutput(const std::string &path, const float *vx, size_t n3) {
    // MPI_MODE_CREATE|MPI_MODE_APPEND then set_view(0): written from offset 0,
    // an existing longer file keeps its tail
    FILE *f = std::fopen(path.c_str(), "r+b");
    if (!f) f = std::fopen(path.c_str(), "wb");
    if (!f) return "cannot open " + path + " for writing";
    bool ok = std::fwrite(vx, sizeof(float), n3, f) == n3;
    ok = (std::fclose(f) == 0) && ok;
    return ok ? "" : "short write to " + path;
}

std::string read_gadget_chunk(const std::string &path, GadgetHeader *h, std::vector<float> *pos,
                              std::vector<float> *vel) {
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) return " cannot read IC file !! " + path;
    int b0 = 0, b1 = 0;
    bool ok = std::fread(&b0, 4, 1, f) == 1 && std::fread(h, sizeof(GadgetHeader), 1, f) == 1 &&
              std::fread(&b1, 4, 1, f) == 1;
    if (!ok) {
        std::fclose(f);
        return "truncated Gadget header " + path;
    }
    const long n = h->npart[1];
    if (n < 0) {
        std::fclose(f);
        return "bad particle count in " + path;
    }
    pos->assign(size_t(3 * n), 0.f);
    vel->assign(size_t(3 * n), 0.f);
    int blk = 0;
    ok = std::fread(&blk, 4, 1, f) == 1 && std::fread(pos->data(), sizeof(float), size_t(3 * n), f) == size_t(3 * n);
    ok = ok && std::fread(&blk, 4, 1, f) == 1 && std::fread(&blk, 4, 1, f) == 1;
    ok = ok && std::fread(vel->data(), sizeof(float), size_t(3 * n), f) == size_t(3 * n);
    std::fclose(f);
    return ok ? "" : "truncated Gadget blocks " + path;
}

}  // namespace ifdm
