// Near-to-far contraction: kernel parameters and launchers (n2f_tc.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/fdtd_b200.h"

namespace fdtd {
namespace n2f {

constexpr int BM = 128;  // directions per CTA (TMEM lanes)
constexpr int BN = 256;  // real accumulator columns per n tile: 32 q x 4 currents x (Re, Im)
constexpr int QT = 32;   // samples q per n tile

struct Face {
    int axis_n, axis_p, axis_q;  // normal and in-face axes (x, y, z = 0, 1, 2)
    int np, nq;                  // samples along p and q
    int ks, nt;                  // K steps and n tiles of the packed operand
    double x_n, o_p, o_q, pitch;
    int64_t b_off, b_freq_stride;  // packed operand: byte offset and per-frequency stride
};

struct Params {
    int n_obs, nfaces;
    const double *dirs;   // [n_obs][3] unit vectors (device)
    const double *freqs;  // [nfreq] (device)
    Face face[6];
    const void *cur[6];   // per face, complex [nfreq][np][nq][4] (device)
    const unsigned char *btiles;
    float2 *partial;      // [nfreq][nfaces][n_obs][4]
    int comp_map[24];     // face-local current -> NL component (Nx Ny Nz Lx Ly Lz)
    uint64_t wait_ns;     // budget of each pipeline wait (0: give up unless already complete)
};

size_t stage_smem(int mode, bool atm);
int b_copy_bytes(int mode);
int k_real_per_step(int mode);
template <typename CT>
cudaError_t launch_pack(int mode, const CT *cur, int nfreq, int np, int nq, int KS, int NT,
                        unsigned char *dst, cudaStream_t st);
cudaError_t launch_contract(int mode, const Params &P, int nfreq, cudaStream_t st);
cudaError_t launch_combine(const Params &P, int nfreq, float2 *nl, cudaStream_t st);
template <typename CT>
cudaError_t launch_fp64(const Params &P, int nfreq, double2 *nl, cudaStream_t st);
int read_error(int reset);
// Wait budget of the contraction kernel's pipeline waits, in nanoseconds;
// a negative value restores the default (0.2 s).  Drain waits keep 0.2 s.
void set_wait_ns(int64_t ns);

}  // namespace n2f
}  // namespace fdtd
