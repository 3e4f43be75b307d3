/*
 * fdtd_b200.h — C ABI of the B200 FDTD engine (libfdtd_b200.so).
 *
 * Plain C: raw device pointers, sizes and scalars; no C++ or torch types.
 * Every entry point returns an FDTD_* status; FDTD_OK == 0.  The message for the
 * last failure on the calling host thread is returned by fdtd_last_error().
 * Launches are asynchronous on the given cudaStream_t (passed as void*, NULL =
 * legacy default stream); nothing here synchronises the device except where a
 * function documents that it returns a host value.
 *
 * Memory layout (all fields, coefficients and ψ stripes): C order, k fastest,
 * idx = (i*Ny + j)*Nz + k, element type double when dtype == FDTD_F64 and float
 * otherwise — the layout of the reference's cl.Buffer objects
 * (opencl_fdtd_solver/engine.py:166-187, yee_update.cl:28).  ψ stripes use the
 * reference face layout (engine.py:290-318): x-normal (2·npml, Ny, Nz),
 * y-normal (Nx, 2·npml, Nz), z-normal (Nx, Ny, 2·npml); low-face layers first.
 *
 * Each declaration names the reference interface it replaces (file:line in the
 * reference project).
 */
#ifndef FDTD_B200_H
#define FDTD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define FDTD_OK 0
#define FDTD_ERR_INVALID 1      /* bad argument: shape, pointer, index, size   */
#define FDTD_ERR_CUDA 2         /* a CUDA runtime call or launch failed        */
#define FDTD_ERR_DEVICE 3       /* a device-side check failed (see flags)      */
#define FDTD_ERR_UNSUPPORTED 4  /* valid request this build/device cannot run  */

#define FDTD_F32 0
#define FDTD_F64 1

#define FDTD_MAX_SOURCES 8      /* pending injections applied by one E launch  */
#define FDTD_MAX_PLANES 4       /* plane DFT monitors fused into one E launch  */
#define FDTD_MAX_FREQS 64       /* frequencies per DFT monitor                 */

/* Grid and time-step scalars.  dtm = dt/mu0, dtm_dl = dt/(mu0*dl),
 * inv_dl = 1/dl, each rounded once to the field dtype by the kernels, as the
 * reference host does (engine.py:541-544, 634). */
typedef struct {
    int32_t nx, ny, nz, npml;
    int32_t dtype;          /* FDTD_F32 or FDTD_F64                            */
    int32_t lossy;          /* nonzero: E = ca*E + ...; zero: ca == 1, not read */
    double dtm, dtm_dl, inv_dl;
    /* x-slab of a grid decomposed along x (x_slab == 0: the whole grid, npml
     * CPML layers on both x faces; the remaining fields are then ignored).
     * x_slab != 0: this grid is one slab; pml_x_lo / pml_x_hi are its x-CPML
     * layers (npml on a global face, else 0), ghost_lo / ghost_hi (0 or 1) mark
     * a ghost plane at local x = 0 / nx-1 that holds a neighbour's plane.  Ghost
     * planes are advanced with boundary-guarded differences and are to be
     * overwritten by the caller's exchange; the x CPML profiles and psi_x stripes
     * ((pml_x_lo + pml_x_hi) x ny x nz) are the slab's own.  No reference
     * counterpart (the reference runs one device). */
    int32_t x_slab, pml_x_lo, pml_x_hi, ghost_lo, ghost_hi, pad_;
} fdtd_grid;

/* Field state.  E/H hold the state at step n (E^n, H^{n-1/2}).
 * E_next/H_next receive the fused step's result and must not alias E/H
 * (the split half-steps update E/H in place and ignore them). */
typedef struct {
    void *E[3];
    void *H[3];
    void *E_next[3];
    void *H_next[3];
    const void *ce[3];      /* dt/(eps0 eps_edge), or cb when lossy            */
    const void *ca[3];      /* read only when grid.lossy != 0                  */
} fdtd_fields;

/* CPML: 1-D b, c and 1/(kappa*dl) for the H (offset 1/2) and E (offset 0)
 * staggers (cpml.py:111-134, engine.py:264-283), and the 12 ψ stripes.
 * psi_h order: Hx_y, Hx_z, Hy_x, Hy_z, Hz_x, Hz_y;
 * psi_e order: Ex_y, Ex_z, Ey_x, Ey_z, Ez_x, Ez_y (yee_update.cl:56-58,176-178).
 * Every entry point updates the ψ stripes in place; psi_h_next is reserved
 * (ignored, may be NULL). */
typedef struct {
    const void *b_h[3], *c_h[3], *ik_h[3];
    const void *b_e[3], *c_e[3], *ik_e[3];
    void *psi_h[6];
    void *psi_h_next[6];
    void *psi_e[6];
} fdtd_cpml;

#define FDTD_SRC_JX 0   /* Ex += -ce_x * amp * w   (sources.cl:26-49)           */
#define FDTD_SRC_EX 1   /* Ex += amp               (sources.cl:7-21)            */

/* One sheet injection on the constant-z plane z, half-open [i0,i1) x [j0,j1).
 * amp is the host-side amplitude after the rim renormalisation of
 * engine.py:512-520; kernels round it to the field dtype. */
typedef struct {
    int32_t kind, z, i0, i1, j0, j1, rim_taper, pad_;
    double amp, rim_edge;
} fdtd_source;

/* A single-plane DFT accumulated in the E epilogue (no reference class; phase
 * convention of monitors.py:571-584).  acc: complex128 (re, im pairs),
 * [ncomp][nfreq][plane cells], components in Ex..Hz bit order of comp_mask,
 * plane cells in C order of the two remaining axes.  phase: device pointer to
 * this step's [nfreq][4] doubles (E re, E im, H re, H im). */
typedef struct {
    int32_t axis, index, comp_mask, nfreq;
    double *acc;
    const double *phase;
} fdtd_plane_dft;

/* ---- Yee time step ------------------------------------------------------- */

/* H half step, in place: H -= dt/mu0 * curl E with CPML (H^{n-1/2} -> H^{n+1/2}).
 * Replaces update_H_interior + update_H_pml (yee_update.cl:11-118) as launched
 * by OpenCLFDTD._update_H (engine.py:540-629). */
int fdtd_update_H(const fdtd_grid *g, const fdtd_fields *f, const fdtd_cpml *c,
                  void *stream);

/* E half step, in place, with pending sheet injections applied to E^n before
 * the update (E = ca*(E + s) + ce*curl H) and plane DFTs of E^{n+1}/H^{n+1/2}.
 * Replaces update_E_interior + update_E_pml (yee_update.cl:120-238) launched
 * by OpenCLFDTD._update_E (engine.py:631-722), preceded by the add_source_*
 * launches made from source callbacks (engine.py:448-538, sources.cl). */
int fdtd_update_E(const fdtd_grid *g, const fdtd_fields *f, const fdtd_cpml *c,
                  const fdtd_source *src, int32_t nsrc,
                  const fdtd_plane_dft *planes, int32_t nplanes, void *stream);

/* One full leapfrog step H -> sources -> E: reads E/H, writes E_next/H_next,
 * ψ stripes in place.  The interior box [npml, N-npml)^3 is updated by one
 * single-pass kernel (H and E per plane, one read and one write of each array);
 * the CPML shell around it: its H by a per-cell kernel on a library-owned side
 * stream (per host thread and device) that overlaps the interior kernel and is
 * joined back by an event, its E afterwards on the caller's stream, as plane
 * marches over the six CPML face slabs (when npml is a multiple of 16 bytes of
 * elements) with the edges and rims per cell on the side stream, or per cell.
 * Replaces the whole of OpenCLFDTD.step() up to the monitors
 * (engine.py:724-735): _update_H, the source callbacks' injections, _update_E. */
int fdtd_step(const fdtd_grid *g, const fdtd_fields *f, const fdtd_cpml *c,
              const fdtd_source *src, int32_t nsrc,
              const fdtd_plane_dft *planes, int32_t nplanes, void *stream);

/* Immediate sheet injection into Ex (used when a source callback reads fields
 * after injecting).  Replaces add_source_Jx / add_source_Ex
 * (sources.cl:7-49, engine.py:448-538). */
int fdtd_add_source(const fdtd_grid *g, void *Ex, const void *ce_x,
                    const fdtd_source *src, void *stream);

/* ---- Huygens-box DFT and far field -------------------------------------- */

/* Box (inclusive indices) and packed face layout x0,x1,y0,y1,z0,z1
 * (monitors.py:396-412). */
typedef struct {
    int32_t ix0, ix1, iy0, iy1, iz0, iz1;
    int32_t off[6];
    int32_t n_face;
    int32_t nfreq;
} fdtd_box;

/* Co-located tangential face DFT at nfreq frequencies, complex128 accumulators
 * acc[6][nfreq][n_face] (Ex..Hz), phase [nfreq][4] for this step.
 * Replaces accumulate_dft_faces_fused (dft_farfield.cl:116-230) launched by
 * OpenCLNear2FarMonitor.__call__ (monitors.py:571-624). */
int fdtd_dft_faces(const fdtd_grid *g, const void *const E[3], const void *const H[3],
                   const fdtd_box *box, double *acc, const double *phase, void *stream);

/* Relative change sqrt(sum|cur-prev|^2 / sum|cur|^2) of one frequency slice
 * over the six face DFTs; writes two doubles (num, den) to out2 (device).
 * scratch: device doubles, at least 2*fdtd_rel_change_blocks(n) of them.
 * Replaces dft_rel_change_partial (dft_farfield.cl:237-290) and the host sum
 * of monitors.py:505-569. */
int fdtd_rel_change_blocks(int32_t n_face);
int fdtd_dft_rel_change(const double *cur, const double *prev, int32_t n_face,
                        int32_t nfreq, int32_t fi, double *scratch, double *out2,
                        void *stream);

/* The same relative change with no device memory supplied by the caller, for
 * callers that must not allocate at run time: drivers that keep the device
 * busy asynchronously (cudaMalloc/cudaFree may synchronise the device and
 * would stall the time-step stream) and hosts whose device memory is a fixed
 * pool set up at start-up.  Its partial sums live in a 16 KiB array inside
 * the library (held on every GPU that loads it until the process exits), so
 * n_face is limited to FDTD_NOALLOC_MAX_FACE; larger boxes get
 * FDTD_ERR_INVALID.  Each call made outside a stream capture looks up that
 * array's device address on the current device (so a device reset cannot
 * leave a stale one); a call inside a capture reuses the device's last
 * address, so make the first call on each device before any stream capture.
 * Calls that overlap on the GPU share the array and race.  No counterpart in
 * the reference. */
#define FDTD_NOALLOC_MAX_FACE (1024 * 256)
int fdtd_dft_rel_change_noalloc(const double *cur, const double *prev, int32_t n_face,
                                int32_t nfreq, int32_t fi, double *out2, void *stream);

/* Far-field E, H at n_obs points (float64 xyz) from face DFT slice fi:
 * eh[n_obs][6] complex128 = (Ex,Ey,Ez,Hx,Hy,Hz); nl_scratch: n_obs*6 complex128.
 * Direct surface sum in float64 with the kernel's sign (eta N_t - r x L).
 * Replaces farfield_accumulate_nl + farfield_nl_to_eh (dft_farfield.cl:372-635)
 * launched by OpenCLNear2FarMonitor.get_farfields (monitors.py:644-731). */
int fdtd_farfield(const fdtd_box *box, const double *acc, int32_t fi, double dl,
                  double k_wave, double eta0, const double *obs_xyz, int32_t n_obs,
                  double *nl_scratch, double *eh, void *stream);

/* Second stage alone: far E, H at n_obs points (float64 xyz, metres) from
 * NL[n_obs][6] = (Nx, Ny, Nz, Lx, Ly, Lz), complex64 (nl_dtype FDTD_F32) or
 * complex128 (FDTD_F64); eh[n_obs][6] complex128.  Replaces farfield_nl_to_eh
 * (dft_farfield.cl:559-635), with the kernel's sign. */
int fdtd_farfield_eh(const void *nl, int32_t nl_dtype, const double *obs_xyz, int32_t n_obs,
                     double k_wave, double eta0, double *eh, void *stream);

/* ---- near-to-far contraction on the tensor cores ------------------------ */
/* NL[f][o][6] = (Nx, Ny, Nz, Lx, Ly, Lz)(r̂_o, f) = Σ_faces Σ_{p,q}
 * e^{+j 2π f r̂_o·r'_{pq}/c0} cur[f][p][q][c], the surface sums that
 * farfield_accumulate_nl (dft_farfield.cl:372-556) forms for one direction at a
 * time, for many directions and frequencies at once.  r'_{pq} is
 * x_n along the face normal and (o_p + p·pitch, o_q + q·pitch) along its two
 * in-face axes (in x, y, z order); cur holds the face's four tangential
 * currents J_p, J_q, M_p, M_q (J = n̂×H, M = −n̂×E) with the quadrature
 * weights already applied.  The far field then follows as in
 * dft_farfield.cl:559-635. */
#define FDTD_N2F_BF16X3 0  /* tcgen05 kind::f16, split BF16 (hi·hi + hi·lo + lo·hi), FP32 accumulate */
#define FDTD_N2F_TF32 1    /* tcgen05 kind::tf32, FP32 accumulate                          */
#define FDTD_N2F_FP64 2    /* float64 direct sum on the CUDA cores (the reference transform) */

typedef struct {
    int32_t normal;        /* axis normal to the face: 0, 1, 2                     */
    int32_t np, nq;        /* samples along the two in-face axes                    */
    int32_t pad_;
    double x_n;            /* face coordinate along its normal (m)                  */
    double o_p, o_q;       /* in-face coordinates of sample (0, 0) (m)              */
    double pitch;          /* sample spacing (m)                                    */
    const void *cur;       /* device, complex [nfreq][np][nq][4] of cur_dtype       */
} fdtd_n2f_face;

/* Workspace bytes fdtd_n2f_contract needs for these faces (0 for FP64). */
int fdtd_n2f_workspace(const fdtd_n2f_face *faces, int32_t nfaces, int32_t nfreq, int32_t n_obs,
                       int32_t mode, uint64_t *bytes);

/* faces: host array of nfaces (1..6) face descriptors; cur_dtype: FDTD_F32
 * (complex64) or FDTD_F64 (complex128); freqs: device, nfreq doubles (Hz);
 * dirs: device, n_obs unit vectors (float64 xyz); nl: device, complex64
 * [nfreq][n_obs][6] for the tensor-core modes, complex128 for FDTD_N2F_FP64.
 * The tensor-core modes pack the currents into the workspace (256-byte
 * aligned), run one CTA per (128 directions, face, frequency) and reduce the
 * faces; bounded waits set bit 1 of fdtd_device_status on timeout. */
int fdtd_n2f_contract(const fdtd_n2f_face *faces, int32_t nfaces, int32_t cur_dtype,
                      const double *freqs, int32_t nfreq, const double *dirs, int32_t n_obs,
                      int32_t mode, void *workspace, uint64_t workspace_bytes, void *nl,
                      void *stream);

/* ---- adjoint (ε-gradient) ------------------------------------------------ */
/* No reference counterpart: the reference has no gradient.  These entry points
 * run the reverse-time sweep of the transposed (discrete adjoint) Yee/CPML
 * step of fdtd_step / fdtd_update_H + fdtd_update_E for a lossless grid
 * (grid.lossy must be 0).  With Ē, H̄ the adjoints of E^{n+1}, H^{n+1/2} and
 * P the adjoints of the ψ recursions, one reverse step is
 *   H̄ += B^T ḡ(Ē, P_E),   P_E' = b_e P_E ± ce Ē          (transposed E update)
 *   Ē += F^T ā(H̄, P_H),   P_H' = b_h P_H ∓ dtm H̄         (transposed H update)
 * where B, F are the backward / forward differences of yee_update.cl:145-150
 * and :30-35 (zero at index 0 / at the last index). */

/* Adjoint state.  The P stripes have the ψ stripe shapes and order of
 * fdtd_cpml and are ping-ponged: a step reads pe/ph and writes pe_next/ph_next
 * (which must not alias them).  With E_next/H_next NULL, E/H are updated in
 * place by one-thread-per-cell kernels.  With all six set (not aliasing E/H),
 * a step reads E/H and writes E_next/H_next: the CPML-free interior runs as one
 * TMA plane march (Ē, H̄, ce read once, Ē', H̄' written once) concurrently with
 * the CPML shell; the caller swaps the buffers after each step.  Both forms
 * give the same values bit for bit. */
typedef struct {
    void *E[3];
    void *H[3];
    const void *pe[6];
    void *pe_next[6];
    const void *ph[6];
    void *ph_next[6];
    const void *ce[3];      /* the forward's dt/(eps0 eps_edge)                */
    void *E_next[3];        /* NULL (in place) or the step's Ē output          */
    void *H_next[3];        /* NULL (in place) or the step's H̄ output          */
} fdtd_adjoint_fields;

/* Adjoint source of a real objective J(D) of plane-DFT samples
 * D[c][f][a][b] = Σ_m phase_m[f] E_c^m over the patch [a0,a1) x [b0,b1) of
 * the plane axis = index (a, b: the two other axes in x, y, z order).
 * seed[c][f][a][b] (complex128) = ∂J/∂Re D + i ∂J/∂Im D, components in
 * Ex, Ey, Ez bit order of comp_mask (E only).  phase: nfreq complex128 values,
 * the phase the forward DFT applied to the E^m this call seeds.  Adds
 * ∂J/∂E^m = Re(seed)·Re(phase) + Im(seed)·Im(phase) to Ē. */
typedef struct {
    int32_t axis, index, a0, a1, b0, b1, comp_mask, nfreq;
    const double *seed;
    const double *phase;
} fdtd_adjoint_seed;

/* Gradient box [lo, hi) of E edges (all three components).  e_next / e_prev
 * are the forward's E^{n+1} and E^n over the box, laid out [3][box cells] in
 * C order (fdtd_capture_box); g[3][box cells] float64 accumulates
 * Σ_n Ē^{n+1}·(E^{n+1} − E^n), which equals ce·∂J/∂ce for a lossless grid,
 * sheet injections included. */
typedef struct {
    int32_t lo[3], hi[3];
    const void *e_next;
    const void *e_prev;
    double *g;
} fdtd_grad_box;

/* Copy E over box [lo, hi) into out ([3][box cells], field dtype). */
int fdtd_capture_box(const fdtd_grid *g, const void *const E[3], const int32_t lo[3],
                     const int32_t hi[3], void *out, void *stream);

/* Ē += ∂J/∂E^m for one seed (used once before the first reverse step). */
int fdtd_adjoint_seed_add(const fdtd_grid *g, void *const Ebar[3],
                          const fdtd_adjoint_seed *seed, void *stream);

/* One reverse step n: on entry Ē = ∂J/∂E^{n+1} (complete), H̄ = ∂J/∂H^{n+1/2}
 * from later steps.  Runs the transposed E update (accumulating gb when
 * non-NULL), then the transposed H update, then adds next_seed (the objective's
 * ∂J/∂E^n, may be NULL).  On return Ē = ∂J/∂E^n and H̄ = ∂J/∂H^{n−1/2}. */
int fdtd_adjoint_step(const fdtd_grid *g, const fdtd_adjoint_fields *a, const fdtd_cpml *c,
                      const fdtd_grad_box *gb, const fdtd_adjoint_seed *next_seed,
                      void *stream);

/* ---- host reads of sub-boxes --------------------------------------------- */

#define FDTD_MAX_REGIONS 32     /* boxes per fdtd_read_regions call            */

/* Half-open cell box [lo, hi) of one field. */
typedef struct {
    int32_t lo[3], hi[3];
} fdtd_region;

/* Copy the cells of nreg boxes of one (nx, ny, nz) field to host memory: the
 * boxes are packed one after another, each in C order, into the device buffer
 * `staging` by one gather launch, then moved to `host` by one device-to-host
 * copy.  Both buffers hold Σ box cells elements of the field dtype.  The copy
 * is asynchronous on `stream` when `host` is pinned; the caller synchronises
 * the stream before reading `host`.  Empty boxes (lo == hi on an axis) are
 * allowed and contribute nothing.  Replaces, for the listed boxes only, the
 * reference's full-volume read of a field (_read_field, engine.py:747-751,
 * behind the Ex…Hz properties, engine.py:767-789), which host monitors such as
 * NumPyNear2FarMonitor.__call__ (monitors.py:229-295) issue every step. */
int fdtd_read_regions(const void *field, int32_t dtype, int32_t nx, int32_t ny, int32_t nz,
                      const fdtd_region *regions, int32_t nreg, void *staging, void *host,
                      void *stream);

/* ---- materials ----------------------------------------------------------- */

/* Yee-edge coefficients from cell-centred εr (and conductivity σ in S/m, may
 * be NULL) computed on the device: ce = (dt/eps0)/ε_edge, or with σ the lossy
 * ca = (1-loss)/(1+loss) and cb = (dt/(eps0 ε_edge))/(1+loss) with
 * loss = (σ_edge dt)/((2 eps0) ε_edge), where ε_edge (σ_edge) is the mean of
 * the two cells sharing the edge and the last plane keeps the cell value.
 * float64 arithmetic in the order of materials.py:28-88, rounded once to the
 * grid dtype, so the result equals set_epsilon's host math (engine.py:212-254)
 * bit for bit.  eps/sigma: nx*ny*nz values of eps_dtype in C order (device).
 * ce receives cb when sigma is given; ca is written only then. */
int fdtd_set_epsilon(const fdtd_grid *g, const void *eps, const void *sigma, int32_t eps_dtype,
                     double dt, double eps0, void *const ce[3], void *const ca[3], void *stream);

/* ---- diagnostics --------------------------------------------------------- */

/* Device time of each launch of fdtd_step, for measurement.  enable != 0 clears
 * the sums and records CUDA events around every launch of each following
 * fdtd_step on its stream; enable == 0 stops recording.  fdtd_profile_read
 * waits for the recorded events and returns the summed milliseconds per
 * launch, [0] CPML-shell H on the side stream (concurrent with [2]), [1] the
 * shell E cells run on the side stream (none unless FDTD_B200_SHELL_SPLIT=1
 * selects that schedule), [2] the interior single-pass kernel, [3] the plane
 * DFT (of the interior cells, or with the face marches of the whole planes),
 * [4] the shell E cells after the join (the face marches and the per-cell
 * edges beside them, or the per-cell kernel with sources and DFTs), and the
 * number of steps recorded.  No reference counterpart. */
int fdtd_profile_steps(int32_t enable);
int fdtd_profile_read(double ms[5], int32_t *nsteps);

/* Number of kernel launches this library has issued since it was loaded. */
int64_t fdtd_launch_count(void);

/* Message for the last non-OK status returned on this host thread. */
const char *fdtd_last_error(void);

/* Device-side error flags raised by kernels since the last reset (bit 0: a
 * bounded wait in the fused step timed out; bit 1: one in the near-to-far
 * contraction did; bit 2: one in the adjoint interior march did).  Synchronises with the device to
 * read the flag; clears it when reset != 0.  No reference counterpart (the
 * reference kernels have no device-side waits). */
int fdtd_device_status(int32_t *flags, int32_t reset);

/* Budget of the bounded pipeline waits of one kernel, for later launches from
 * this process: kernel FDTD_WAIT_INTERIOR (the fused step's interior kernel,
 * its CPML face marches and the adjoint interior march; budget in mbarrier
 * polls, default and maximum 2^24) or FDTD_WAIT_N2F (the
 * tensor-core near-to-far contraction; budget in nanoseconds, default 2e8).
 * budget < 0 restores the default; 0 makes a wait give up unless its phase has
 * already completed, which exercises the timeout path: the kernel raises its
 * fdtd_device_status bit, still waits (with the default bound) for every copy
 * and MMA it issued, frees what it holds and returns.  A launch that timed out
 * leaves its outputs undefined.  No reference counterpart. */
#define FDTD_WAIT_INTERIOR 0
#define FDTD_WAIT_N2F 1
int fdtd_set_wait_budget(int32_t kernel, int64_t budget);

/* Library build tag, e.g. "fdtd_b200 sm_100a". */
const char *fdtd_version(void);

#ifdef __cplusplus
}
#endif
#endif /* FDTD_B200_H */
