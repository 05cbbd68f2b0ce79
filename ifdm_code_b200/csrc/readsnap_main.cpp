// readsnap -- a z-slice of a snapshot as text (the reference's
// src/readsnap.cpp, same command line, output file and line format).
//
//   readsnap N zslice t opath icpath
//
// reads <opath>/output<t>.dat (f64 mfdm, f64 g, f64 a, f64 x[N], c128 psi[N^3],
// z fastest) and writes <icpath>/output<t>.dat.z<zslice> with one line per
// (i, j):  x[i] x[j] |psi|^2 m  arg(psi)  for psi = psi[(i N + j) N + zslice]
// and m = mfdm[eV] * 1.783e-36 / 1.989e30 (solar masses), formatted by the
// default iostream rules.  Only the N^2 values of the slice are read (one
// positioned read per row instead of the whole N^3 array).
//
// Behaviour kept from the reference: a wrong argument count prints
// "ERROR: Arguments <argc>!= 5" and exits 0; an unreadable input prints
// "ERROR: cant read binary file !!" and the slice is written from zeros
// (the reference prints its uninitialised header there; this tool prints 0).
#include <fcntl.h>
#include <unistd.h>

#include <cmath>
#include <complex>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

static bool read_at(int fd, void *dst, size_t n, off_t off) {
    char *p = static_cast<char *>(dst);
    while (n > 0) {
        const ssize_t r = pread(fd, p, n, off);
        if (r <= 0) return false;
        p += r;
        n -= size_t(r);
        off += r;
    }
    return true;
}

int main(int argc, char **argv) {
    if (argc != 6) {
        std::cout << "ERROR: Arguments " << argc << "!= 5 \n";
        return 0;
    }
    const int N = std::atoi(argv[1]);
    const int zslice = std::atoi(argv[2]);
    const int t = std::atoi(argv[3]);
    const std::string opath = argv[4], icpath = argv[5];
    const double kg2eV = 1.783e-36, kg2solar = 1.989e30;

    const std::string in_name = opath + "/output" + std::to_string(t) + ".dat";
    const std::string out_name = icpath + "/output" + std::to_string(t) + ".dat.z" + std::to_string(zslice);
    std::ofstream ofile(out_name);

    double hdr[3] = {0, 0, 0};
    std::vector<double> x(N > 0 ? N : 0, 0.0);
    std::vector<std::complex<double>> slice(size_t(N > 0 ? N : 0) * (N > 0 ? N : 0));
    const int fd = open(in_name.c_str(), O_RDONLY);
    if (fd >= 0 && N > 0 && zslice >= 0 && zslice < N) {
        bool ok = read_at(fd, hdr, sizeof hdr, 0) && read_at(fd, x.data(), N * sizeof(double), sizeof hdr);
        const off_t psi0 = off_t(3 + N) * sizeof(double);
        for (size_t r = 0; ok && r < size_t(N) * N; ++r)
            ok = read_at(fd, &slice[r], sizeof(std::complex<double>),
                         psi0 + off_t((r * N + zslice) * sizeof(std::complex<double>)));
        if (!ok) std::cout << "ERROR: cant read binary file !!\n";
    } else {
        std::cout << "ERROR: cant read binary file !!\n";
    }
    if (fd >= 0) close(fd);

    double mfdm = hdr[0];
    std::cout << "writing snapshot mfdm = " << mfdm << " and g = " << hdr[1] << " at a = " << hdr[2] << "\n";
    std::cout << "input file = " << in_name << "\n output file = " << out_name << "\n";
    mfdm *= kg2eV / kg2solar;
    if (ofile) {
        for (int i = 0; i < N; ++i)
            for (int j = 0; j < N; ++j) {
                const std::complex<double> v = slice[size_t(i) * N + j];
                std::ostringstream line;
                line << x[i] << " " << x[j] << " " << std::pow(std::abs(v), 2) * mfdm << " " << std::arg(v) << "\n";
                ofile << line.str();
            }
    }
    return 0;
}
