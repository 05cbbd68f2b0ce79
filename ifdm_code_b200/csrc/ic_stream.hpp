// ic_stream.hpp -- Gadget chunk files streamed to the device.
//
// The reference reads each chunk whole into host vectors
// (:412-545).  Here every position and velocity block is cut into byte
// ranges that up to 16 threads read side by side, each in pieces through two
// pinned buffers: while one piece is copied to the device (asynchronous, on
// the thread's own stream) the next is read.  Particles land directly at
// their place in the device arrays, in the order the one-rank reference
// processes them:
//
//   per chunk c:  [ghosts: its last lg_c particles] [its n_c particles] [one zero particle]
//
// (ref1 mode: particles beyond the last cell centre are rank 0's left ghosts
// and its own, src/gadget_IC.h:445-448,:496-502; the extra zero particle is
// numpart + 1, :431-432), or just [n_c particles] per chunk (exact mode).
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "io.hpp"

namespace ifdm {

struct IcChunk {
    std::string path;
    GadgetHeader h{};
    long n = 0;     // particles in the file
    long lg = 0;    // trailing particles copied in front as ghosts (ref1)
    long base = 0;  // first particle slot of this chunk in the device arrays
};

// Headers of <icpath>.0 .. .<nchunks-1>, in order (the first problem found
// is returned: missing file, truncated header or blocks); with ref1 the ghost
// counts from the tail of each chunk's positions (N cells across BoxSize).
// np_total receives the particle slots of the device arrays.
std::string ic_scan_chunks(const std::string &icpath, int nchunks, int N, bool ref1, std::vector<IcChunk> *out,
                           long *np_total);

// Fills d_pos / d_vel (3 floats per particle slot) from the files.  Returns
// when the copies are complete.  piece_bytes: the size of one read (each
// worker pins two of them).
std::string ic_upload(const std::vector<IcChunk> &chunks, bool ref1, float *d_pos, float *d_vel, int device,
                      size_t piece_bytes = size_t(8) << 20);

}  // namespace ifdm
