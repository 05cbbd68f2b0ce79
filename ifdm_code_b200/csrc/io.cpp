// io.cpp -- snapshot and voutput I/O (formats in io.hpp; Gadget chunks are read by ic_stream.cpp).
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

}  // namespace ifdm
