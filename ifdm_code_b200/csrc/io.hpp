// io.hpp -- the reference's file formats.
//
//  snapshot  <opath>output<t>.dat (src/write3D.h:7-22, :55-77, :86-97):
//            f64 mfdm [eV], f64 g*cm2Mpc^3 [eV cm^3], f64 a, f64 x[N],
//            complex128 psi[N][N][N] (z fastest); read back by read_rerun
//            (src/gadget_IC.h:709-750) at offset (N+3)*8.
//  voutput   <opath>voutput.dat: f32 v_x[N^3] written at the IC
//            (src/write3D.h:24-53), at offset 0 of an existing file.
//  Gadget-1  <icpath>.<c>, c = 0..3: int 256, io_header (256 B), int 256,
//            int, f32 pos[3n], int, int, f32 vel[3n], int ...
//            (src/gadget_IC.h:17-33, :259-353).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace ifdm {

struct GadgetHeader {  // src/gadget_IC.h:17-33
    int npart[6];
    double mass[6];
    double time;
    double redshift;
    int flag_sfr;
    int flag_feedback;
    int npartTotal[6];
    int flag_cooling;
    int num_files;
    double BoxSize;
    double Omega0;
    double OmegaLambda;
    double HubbleParam;
    char fill[256 - 6 * 4 - 6 * 8 - 2 * 8 - 2 * 4 - 6 * 4 - 2 * 4 - 4 * 8];
};
static_assert(sizeof(GadgetHeader) == 256, "Gadget header must be 256 bytes");

std::string snapshot_path(const std::string &prefix, int t);

// Header + psi.  psi: N^3 complex128 interleaved.  Returns "" or an error.
std::string write_snapshot(const std::string &path, double mfdm, double g_cm3, double a, const std::vector<double> &x,
                           const double *psi, size_t n3);
// Reads a, x and psi of an N^3 snapshot (psi may be null to read the header only).
std::string read_snapshot(const std::string &path, int N, double *a, std::vector<double> *x, double *psi);
std::string write_voutput(const std::string &path, const float *vx, size_t n3);

}  // namespace ifdm
