/*
 * krakenb200.h -- C ABI of the B200 stream-collide library (libkrakenb200.so).
 *
 * Each entry point replaces one Kraken.jl kernel wrapper on its
 * stream-collide path; the comment above it cites the reference function
 * (file:line, paths inside the Kraken.jl repository) whose argument meaning
 * and error behaviour it keeps.  A Julia backend binds these with `ccall`
 * (krakenn.jl_b200/julia/KrakenB200.jl); the Python host layer in
 * krakenn.jl_b200/ binds them with ctypes.
 *
 * Conventions shared by every entry point
 *   - Arrays are raw DEVICE pointers owned by the caller, in Julia
 *     column-major order with 0-based indices:
 *        D2Q9   f[i + Nx*(j + Ny*q)],         fields  a[i + Nx*j]
 *        D3Q19  f[i + Nx*(j + Ny*(k + Nz*q))], fields  a[i + Nx*(j + Ny*k)]
 *     (q is the reference's population index minus one).  A CuArray of
 *     size (Nx, Ny, 9) passes its pointer unchanged.
 *   - Masks (`is_solid`) are one byte per node (Julia Bool); NULL means "no
 *     solid node", which skips the mask read.
 *   - `dtype` selects the population storage (kb_dtype).  Macroscopic
 *     fields (rho, ux, ...) are double for KB_F64 and float otherwise.
 *   - `stream` is a cudaStream_t (NULL = legacy default stream).  Calls are
 *     stream-ordered and asynchronous; nothing synchronises unless the entry
 *     point says so.  There are no internal host threads.
 *   - Return value: KB_OK (0) or a negative kb_status.  The message of the
 *     last failure on the calling thread is kb_last_error().  There is no
 *     fallback: an unsupported combination is an error, never a CPU path.
 *   - Operations are in place (the reference's `!` functions); the caller
 *     swaps f_in/f_out between steps, as the reference drivers do.
 */
#ifndef KRAKENB200_H
#define KRAKENB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    KB_OK = 0,
    KB_ERR_ARG = -1,         /* bad pointer, size or parameter              */
    KB_ERR_UNSUPPORTED = -2, /* dtype / option not available for this op    */
    KB_ERR_CUDA = -3,        /* a CUDA call failed (message says which)     */
    KB_ERR_TIMEOUT = -4,     /* a bounded device wait ran out               */
    KB_ERR_NONFINITE = -5,   /* a reduction met NaN or Inf                  */
    KB_ERR_NOMEM = -6        /* device allocation of a handle failed        */
} kb_status;

typedef enum {
    KB_F64 = 0,      /* double populations (reference Float64 semantics)   */
    KB_F32 = 1,      /* float populations (reference Float32 semantics)    */
    KB_F32_DEV = 2,  /* float deviations f - w_q, FP32 collision           */
    KB_F16_DEV = 3,  /* IEEE half deviations f - w_q, FP32 collision       */
    KB_BF16_DEV = 4, /* bfloat16 deviations f - w_q, FP32 collision        */
    /* Same memory format as KB_F16_DEV / KB_BF16_DEV; kernels that write them
     * round stochastically (sm_100a cvt.rs), so the rounding error has zero
     * mean.  Only kb_fused_trt_step_3d writes them; everything that reads
     * populations accepts them. */
    KB_F16_DEV_SR = 5,
    KB_BF16_DEV_SR = 6
} kb_dtype;

/* Library version string ("krakenb200 <semver> sm_100a"). */
const char *kb_version(void);
/* Message of the last error on the calling thread ("" if none). */
const char *kb_last_error(void);
/* Block until all work queued on `stream` is done; reports any pending
 * asynchronous CUDA error.  KernelAbstractions.synchronize(backend). */
int kb_sync(void *stream);

/* ---------------------------------------------------------------- D2Q9 -- */

/* stream_2d!(f_out, f_in, Nx, Ny)  -- src/kernels/collide_stream_2d.jl:77 */
int kb_stream_2d(void *f_out, const void *f_in, int Nx, int Ny, int dtype, void *stream);

/* collide_2d!(f, is_solid, omega)  -- src/kernels/collide_stream_2d.jl:96 */
int kb_collide_2d(void *f, const uint8_t *is_solid, int Nx, int Ny, double omega, int dtype,
                  void *stream);

/* apply_zou_he_north_2d!(f, u_wall_x, Nx, Ny) -- src/kernels/boundary_2d.jl:56 */
int kb_apply_zou_he_north_2d(void *f, double u_wall_x, int Nx, int Ny, int dtype, void *stream);

/* apply_zou_he_south_2d!(f, u_wall_x, Nx) -- src/kernels/boundary_2d.jl:163 */
int kb_apply_zou_he_south_2d(void *f, double u_wall_x, int Nx, int Ny, int dtype, void *stream);

/* apply_zou_he_west_2d!(f, u_in, Nx, Ny) -- src/kernels/boundary_2d.jl:198 */
int kb_apply_zou_he_west_2d(void *f, double u_in, int Nx, int Ny, int dtype, void *stream);

/* apply_zou_he_pressure_east_2d!(f, Nx, Ny; rho_out) -- src/kernels/boundary_2d.jl:237 */
int kb_apply_zou_he_pressure_east_2d(void *f, int Nx, int Ny, double rho_out, int dtype,
                                     void *stream);

/* apply_zou_he_pressure_west_2d!(f, Nx, Ny; rho_in) -- src/kernels/boundary_2d.jl:295 */
int kb_apply_zou_he_pressure_west_2d(void *f, int Nx, int Ny, double rho_in, int dtype,
                                     void *stream);

/* apply_extrapolate_east_2d!(f, Nx, Ny) -- src/kernels/boundary_2d.jl:319 */
int kb_apply_extrapolate_east_2d(void *f, int Nx, int Ny, int dtype, void *stream);

/* apply_bounce_back_wall_2d!(f, Nx, Ny, side) -- src/kernels/boundary_2d.jl:117.
 * wall_id: 1 south, 2 west, 3 east, 4 north (the reference's Int32 codes). */
int kb_apply_bounce_back_wall_2d(void *f, int Nx, int Ny, int wall_id, int dtype, void *stream);

/* f[.., q] = equilibrium(D2Q9(), rho, ux, uy, q) at every node
 *   -- src/lattice/d2q9.jl:60-67, as the initialisers of src/drivers/basic.jl:265
 * fill f.  Fields are double (fields_dtype KB_F64) or float (KB_F32), of
 * Nx*Ny nodes each; populations are KB_F64 or KB_F32. */
int kb_init_equilibrium_2d(void *f, const void *rho, const void *ux, const void *uy,
                           int fields_dtype, int Nx, int Ny, int dtype, void *stream);

/* compute_macroscopic_2d!(rho, ux, uy, f) -- src/kernels/macroscopic.jl:32 */
int kb_compute_macroscopic_2d(void *rho, void *ux, void *uy, const void *f, int Nx, int Ny,
                              int dtype, void *stream);

/* compute_macroscopic_forced_2d!(rho, ux, uy, f, Fx, Fy)
 *   -- src/kernels/macroscopic.jl:84-118: u = (sum c f + F/2) / rho */
int kb_compute_macroscopic_forced_2d(void *rho, void *ux, void *uy, const void *f, int Nx, int Ny,
                                     double Fx, double Fy, int dtype, void *stream);

/* fused_bgk_step!(f_out, f_in, rho, ux, uy, is_solid, Nx, Ny, omega)
 *   -- src/kernels/fused_bgk_2d.jl:67 */
int kb_fused_bgk_step(void *f_out, const void *f_in, void *rho, void *ux, void *uy,
                      const uint8_t *is_solid, int Nx, int Ny, double omega, int dtype,
                      void *stream);

/* trt_rates(nu; Lambda) -> (s_plus, s_minus) -- src/kernels/fused_trt_2d.jl:129 */
int kb_trt_rates(double nu, double Lambda, double *s_plus, double *s_minus);

/* fused_trt_step!(f_out, f_in, rho, ux, uy, is_solid, Nx, Ny, nu; Lambda)
 *   -- src/kernels/fused_trt_2d.jl:145 */
int kb_fused_trt_step(void *f_out, const void *f_in, void *rho, void *ux, void *uy,
                      const uint8_t *is_solid, int Nx, int Ny, double nu, double Lambda, int dtype,
                      void *stream);

/* collide_guo_2d!(f, is_solid, omega, Fx, Fy) -- src/kernels/collide_guo_2d.jl:5-90:
 * in-place BGK with the Guo source of a constant body force.
 * The forced collisions (kb_collide_guo_*, kb_collide_boussinesq_2d/_3d) in
 * KB_F64 give the reference arithmetic bit for bit.  In KB_F32, on an even Nx
 * with 8-byte aligned fields (2-byte aligned mask), two adjacent nodes are
 * updated per thread in packed FP32x2 round-to-nearest arithmetic: the same
 * operations, within 3 ulp of the one-node form. */
int kb_collide_guo_2d(void *f, const uint8_t *is_solid, int Nx, int Ny, double omega, double Fx,
                      double Fy, int dtype, void *stream);

/* collide_guo_field_2d!(f, is_solid, Fx_field, Fy_field, omega)
 *   -- src/kernels/collide_guo_2d.jl:93-162: per-node force (fields of the
 * population's type). */
int kb_collide_guo_field_2d(void *f, const uint8_t *is_solid, const void *Fx_field,
                            const void *Fy_field, int Nx, int Ny, double omega, int dtype,
                            void *stream);

/* fused_trt_libb_v2_step!(f_out, f_in, rho, ux, uy, is_solid, q_wall,
 *   uw_link_x, uw_link_y, Nx, Ny, nu; Lambda) -- src/kernels/li_bb_2d_v2.jl:35-41,
 * 104-115: pull with half-way bounce-back, rest equilibrium on solid nodes,
 * Bouzidi interpolated bounce-back of every cut link before the TRT
 * collision (ApplyLiBBPrePhase, src/kernels/dsl/bricks.jl:516-560).
 * q_wall / uw_link_x / uw_link_y: per-link arrays laid out like f (9
 * planes, the population's type).  rho/ux/uy: all or none (NULL).
 * KB_F64 / KB_F32. */
int kb_fused_trt_libb_step(void *f_out, const void *f_in, void *rho, void *ux, void *uy,
                           const uint8_t *is_solid, const void *q_wall, const void *uw_link_x,
                           const void *uw_link_y, int Nx, int Ny, double nu, double Lambda,
                           int dtype, void *stream);

/* In-place A-A streaming on one population buffer, the scheme of
 * aa_even_step!/aa_odd_step! (src/kernels/aa_bgk_2d.jl:125,138).  Those
 * reference kernels let neighbouring nodes read and write the same slot in
 * one launch, so their result depends on execution order; these two do not.
 * Buffer states: S (slot qb(x) holds the post-collision f_q(x)) and P
 * (slot q(x) holds the f_q arriving at x).  kb_aa_stream_step_2d takes S to
 * P, kb_aa_local_step_2d takes P to S; each is one BGK step with half-way
 * bounce-back and the solid swap.  A pull-format buffer with slots q and qb
 * swapped is state S, and a stream step followed by a local step equals two
 * kb_fused_bgk_step calls bit for bit.  rho/ux/uy: all NULL or all set. */
int kb_aa_stream_step_2d(void *f, void *rho, void *ux, void *uy, const uint8_t *is_solid, int Nx,
                         int Ny, double omega, int dtype, void *stream);
int kb_aa_local_step_2d(void *f, void *rho, void *ux, void *uy, const uint8_t *is_solid, int Nx,
                        int Ny, double omega, int dtype, void *stream);

/* collide_mrt_2d!(f, is_solid, nu; s_e, s_eps, s_q) -- src/kernels/collide_mrt_2d.jl:118 */
int kb_collide_mrt_2d(void *f, const uint8_t *is_solid, int Nx, int Ny, double nu, double s_e,
                      double s_eps, double s_q, int dtype, void *stream);

/* stream_fully_periodic_2d!(f_out, f_in, Nx, Ny) -- src/kernels/stream_periodic_2d.jl:112 */
int kb_stream_fully_periodic_2d(void *f_out, const void *f_in, int Nx, int Ny, int dtype,
                                void *stream);

/* stream_periodic_x_wall_y_2d!(f_out, f_in, Nx, Ny) -- src/kernels/stream_periodic_2d.jl:71 */
int kb_stream_periodic_x_wall_y_2d(void *f_out, const void *f_in, int Nx, int Ny, int dtype,
                                   void *stream);

/* One cavity step of run_cavity_2d (src/drivers/basic.jl:121-136) in ONE
 * launch: stream_2d! -> apply_zou_he_north_2d! -> collide_2d! ->
 * compute_macroscopic_2d!.  Every stage is node-local after the pull, so the
 * fused step gives the same bits as the four reference launches. */
int kb_cavity_step_2d(void *f_out, const void *f_in, void *rho, void *ux, void *uy,
                      const uint8_t *is_solid, int Nx, int Ny, double omega, double u_lid,
                      int dtype, void *stream);

/* One consistent-initialisation iteration for the MRT cavity: the step of
 * kb_cavity_mrt_step_2d with the collision's velocity held at the given field
 * (ux, uy; double or float by fields_dtype) and the momentum reset to rho*u.
 * Repeating it from f = equilibrium(rho, u) makes rho and the
 * non-equilibrium populations consistent with u (Mei, Luo, Lallemand and
 * d'Humieres 2006).  The warm start runs a few hundred of these before the
 * plain steps.  No reference counterpart. */
int kb_cavity_mrt_init_step_2d(void *f_out, const void *f_in, const void *ux, const void *uy,
                               int fields_dtype, const uint8_t *is_solid, int Nx, int Ny, double nu,
                               double s_e, double s_eps, double s_q, double u_lid, int dtype,
                               void *stream);

/* Lid-driven cavity step with a moving-wall half-way bounce-back lid: the
 * fused pull + half-way bounce-back + BGK + moments of fused_bgk_step!
 * (src/kernels/fused_bgk_2d.jl:8-59) with the lid link rule of
 * ApplyHalfwayBBPrePhase (src/kernels/dsl/bricks.jl:447-487) on the top row's
 * north-pointing links, wall velocity (u_lid, 0).  Moments (pre-collision)
 * are written when rho/ux/uy are given (all or none). */
int kb_cavity_movingwall_step_2d(void *f_out, const void *f_in, void *rho, void *ux, void *uy,
                                 const uint8_t *is_solid, int Nx, int Ny, double omega,
                                 double u_lid, int dtype, void *stream);

/* One step of the MRT cavity loop of test/test_mrt.jl:19-25 (stream_2d! ->
 * apply_zou_he_north_2d! -> collide_mrt_2d!(f, is_solid, nu; s_e, s_eps,
 * s_q) -> compute_macroscopic_2d!) in one launch, same bits.  rho/ux/uy:
 * all NULL (moments skipped) or all set. */
int kb_cavity_mrt_step_2d(void *f_out, const void *f_in, void *rho, void *ux, void *uy,
                          const uint8_t *is_solid, int Nx, int Ny, double nu, double s_e,
                          double s_eps, double s_q, double u_lid, int dtype, void *stream);

/* fused_natconv_step!(f_out, f_in, g_out, g_in, Temp, Nx, Ny, omega_f,
 *   omega_T, beta_g, T_ref_buoy, T_hot, T_cold) -- src/kernels/fused_thermal_2d.jl:251
 * KB_F64 / KB_F32 keep the reference arithmetic (f, g and Temp of that type).
 * The deviation storages (KB_F32_DEV, KB_F16_DEV, KB_BF16_DEV and the
 * stochastic-rounding 16-bit codes) hold f - w_q and g - w_q * T_ref_buoy in
 * that type and step in FP32; Temp is then float.  Same for the _vt_ step. */
int kb_fused_natconv_step(void *f_out, const void *f_in, void *g_out, const void *g_in,
                          void *Temp, int Nx, int Ny, double omega_f, double omega_T,
                          double beta_g, double T_ref_buoy, double T_hot, double T_cold,
                          int dtype, void *stream);

/* fused_natconv_vt_step!(..., nu_ref, T0_visc, alpha_visc, omega_T, beta_g,
 *   T_ref_buoy, T_hot, T_cold) -- src/kernels/fused_thermal_2d.jl:268 */
int kb_fused_natconv_vt_step(void *f_out, const void *f_in, void *g_out, const void *g_in,
                             void *Temp, int Nx, int Ny, double nu_ref, double T0_visc,
                             double alpha_visc, double omega_T, double beta_g, double T_ref_buoy,
                             double T_hot, double T_cold, int dtype, void *stream);

/* compute_temperature_2d!(Temp, g) -- src/kernels/thermal_2d.jl:113 */
int kb_compute_temperature_2d(void *Temp, const void *g, int Nx, int Ny, int dtype, void *stream);

/* Unfused thermal DDF (the reference's Rayleigh-Benard loop,
 * src/drivers/thermal.jl:101-130).  Fields have the population's type.
 * Faces: 0 west, 1 east, 2 south, 3 north. */

/* collide_thermal_2d!(g, ux, uy, omega_T) -- src/kernels/thermal_2d.jl:16-81 */
int kb_collide_thermal_2d(void *g, const void *ux, const void *uy, int Nx, int Ny, double omega_T,
                          int dtype, void *stream);

/* collide_thermal_masked_2d!(g, ux, uy, omega_T, is_skip)
 *   -- src/kernels/thermal_2d.jl:83-109; is_skip NULL skips no node */
int kb_collide_thermal_masked_2d(void *g, const void *ux, const void *uy, const uint8_t *is_skip,
                                 int Nx, int Ny, double omega_T, int dtype, void *stream);

/* _fixed_temp_{west,east,south,north}_2d!(g, T_wall, ..., T_c, skip_c)
 *   -- src/kernels/thermal_2d.jl:174-350.  Half-way anti-bounce-back on one
 * face of the post-stream array; the face's two corner slots (low / high end
 * of the face) take T_corner_* and are left alone when skip_* is non-zero.
 * apply_fixed_temp_<face>_2d!(g, T_wall, ...) is T_corner_* = T_wall,
 * skip_* = 0.  Call once per step. */
int kb_apply_fixed_temp_face_2d(void *g, int Nx, int Ny, int face, double T_wall,
                                double T_corner_lo, double T_corner_hi, int skip_lo, int skip_hi,
                                int dtype, void *stream);

/* apply_fixed_temp_2d!(g, Nx, Ny; west, east, south, north)
 *   -- src/kernels/thermal_2d.jl:371-417.  faces: bit n set = face n is
 * Dirichlet at T_faces[n] (T_faces has 4 entries, W E S N).  A corner slot
 * shared by two Dirichlet faces is flipped once, with the mean temperature.
 * One launch. */
int kb_apply_fixed_temp_2d(void *g, int Nx, int Ny, unsigned faces, const double *T_faces,
                           int dtype, void *stream);

/* collide_boussinesq_2d!(f, Temp, is_solid, omega, beta_g, T_ref)
 *   -- src/kernels/thermal_2d.jl:421-473, 573-579 */
int kb_collide_boussinesq_2d(void *f, const void *Temp, const uint8_t *is_solid, int Nx, int Ny,
                             double omega, double beta_g, double T_ref, int dtype, void *stream);

/* collide_boussinesq_vt_2d!(f, Temp, is_solid, nu_ref, T_ref, A_arr, beta_g)
 *   -- src/kernels/thermal_2d.jl:482-559 (Arrhenius nu(T)) */
int kb_collide_boussinesq_vt_2d(void *f, const void *Temp, const uint8_t *is_solid, int Nx, int Ny,
                                double nu_ref, double T_ref, double A_arr, double beta_g,
                                int dtype, void *stream);

/* collide_boussinesq_vt_modified_2d!(f, Temp, is_solid, nu_ref, T0_visc,
 *   alpha_visc, beta_g, T_ref_buoy) -- src/kernels/thermal_2d.jl:593-670 */
int kb_collide_boussinesq_vt_modified_2d(void *f, const void *Temp, const uint8_t *is_solid,
                                         int Nx, int Ny, double nu_ref, double T0_visc,
                                         double alpha_visc, double beta_g, double T_ref_buoy,
                                         int dtype, void *stream);

/* --------------------------------------------------------------- D3Q19 -- */

/* stream_3d!(f_out, f_in, Nx, Ny, Nz) -- src/kernels/collide_stream_3d.jl:119 */
int kb_stream_3d(void *f_out, const void *f_in, int Nx, int Ny, int Nz, int dtype, void *stream);

/* collide_3d!(f, is_solid, omega) -- src/kernels/collide_stream_3d.jl:137 */
int kb_collide_3d(void *f, const uint8_t *is_solid, int Nx, int Ny, int Nz, double omega,
                  int dtype, void *stream);

/* _apply_zou_he_velocity_3d!(f, face, idx_fixed, u_n, u_t1, u_t2)
 *   -- src/kernels/boundary_3d.jl:154-223, 300-305.
 * face: 0 west, 1 east, 2 south, 3 north, 4 bottom, 5 top; the fixed index
 * is the face's own (0 or N-1). */
int kb_apply_zou_he_velocity_3d(void *f, int Nx, int Ny, int Nz, int face, double u_normal,
                                double u_tang1, double u_tang2, int dtype, void *stream);

/* apply_zou_he_top_3d!(f, u_wall_x, Nx, Ny, Nz) -- src/kernels/boundary_3d.jl:326 */
int kb_apply_zou_he_top_3d(void *f, double u_wall_x, int Nx, int Ny, int Nz, int dtype,
                           void *stream);

/* _apply_zou_he_pressure_3d!(f, face, idx_fixed, rho_out)
 *   -- src/kernels/boundary_3d.jl:232-288, 307-312 */
int kb_apply_zou_he_pressure_3d(void *f, int Nx, int Ny, int Nz, int face, double rho_out,
                                int dtype, void *stream);

/* compute_macroscopic_3d!(rho, ux, uy, uz, f) -- src/kernels/macroscopic.jl:75 */
int kb_compute_macroscopic_3d(void *rho, void *ux, void *uy, void *uz, const void *f, int Nx,
                              int Ny, int Nz, int dtype, void *stream);

/* compute_macroscopic_forced_3d!(rho, ux, uy, uz, f, Fx, Fy, Fz)
 *   -- src/kernels/macroscopic.jl:121-160 */
int kb_compute_macroscopic_forced_3d(void *rho, void *ux, void *uy, void *uz, const void *f,
                                     int Nx, int Ny, int Nz, double Fx, double Fy, double Fz,
                                     int dtype, void *stream);

/* compute_macroscopic_forced_field_3d!(rho, ux, uy, uz, f, Fx, Fy, Fz) with
 * per-node force fields -- src/kernels/macroscopic.jl:164-200 */
int kb_compute_macroscopic_forced_field_3d(void *rho, void *ux, void *uy, void *uz, const void *f,
                                           const void *Fx_field, const void *Fy_field,
                                           const void *Fz_field, int Nx, int Ny, int Nz,
                                           int dtype, void *stream);

/* stream_periodic_xz_wall_y_3d!(f_out, f_in, Nx, Ny, Nz)
 *   -- src/kernels/stream_periodic_3d.jl:24-92: x and z wrap, half-way
 * bounce-back on the y faces */
int kb_stream_periodic_xz_wall_y_3d(void *f_out, const void *f_in, int Nx, int Ny, int Nz,
                                    int dtype, void *stream);

/* Ghost planes of a z-slab of D3Q19 populations f[q][k][j][i] with nz_alloc
 * planes (a ghost plane at k = 0 if lo, at k = nz_alloc - 1 if hi) whose
 * neighbouring slabs are the slab itself, i.e. one rank on a periodic z
 * axis: the c_z = +1 populations (5, 11, 12, 15, 16) of the top real plane
 * fill the bottom ghost, the c_z = -1 populations (6, 13, 14, 17, 18) of the
 * first real plane fill the top ghost.  Between ranks the same planes travel
 * by point-to-point messages.  No reference counterpart: the reference runs
 * one grid on one device. */
int kb_slab_fill_ghosts_3d(void *f, int Nx, int Ny, int nz_alloc, int lo, int hi, int dtype,
                           void *stream);

/* Unfused thermal DDF in 3D (run_natural_convection_3d,
 * src/drivers/thermal.jl:455-537).  Fields have the population's type. */

/* collide_thermal_3d!(g, ux, uy, uz, omega_T) -- src/kernels/thermal_3d.jl:12-124 */
int kb_collide_thermal_3d(void *g, const void *ux, const void *uy, const void *uz, int Nx, int Ny,
                          int Nz, double omega_T, int dtype, void *stream);

/* compute_temperature_3d!(Temp, g) -- src/kernels/thermal_3d.jl:128-155 */
int kb_compute_temperature_3d(void *Temp, const void *g, int Nx, int Ny, int Nz, int dtype,
                              void *stream);

/* _fixed_temp_{west,...,top}_3d!(g, T_wall, ..., T_e, skip_e)
 *   -- src/kernels/thermal_3d.jl:193-480.  Half-way anti-bounce-back on one
 * face (0 west .. 5 top) of the post-stream array.  Edge slot n (the face's
 * first in-plane axis low / high, then the second low / high: (y, z) for
 * x-faces, (x, z) for y-faces, (x, y) for z-faces) takes T_edge[n] (NULL:
 * T_wall) and is left alone when bit n of skip_edges is set.
 * apply_fixed_temp_<face>_3d!(g, T_wall, ...) is T_edge = NULL, skip 0. */
int kb_apply_fixed_temp_face_3d(void *g, int Nx, int Ny, int Nz, int face, double T_wall,
                                const double *T_edge, unsigned skip_edges, int dtype,
                                void *stream);

/* apply_fixed_temp_3d!(g, Nx, Ny, Nz; west, east, south, north, bottom, top)
 *   -- src/kernels/thermal_3d.jl:494-553.  faces: bit n set = face n is
 * Dirichlet at T_faces[n] (6 entries).  An edge slot shared by two
 * Dirichlet faces is flipped once, with the mean temperature.  One launch. */
int kb_apply_fixed_temp_3d(void *g, int Nx, int Ny, int Nz, unsigned faces, const double *T_faces,
                           int dtype, void *stream);

/* collide_boussinesq_3d!(f, Temp, is_solid, omega, beta_g, T_ref)
 *   -- src/kernels/thermal_3d.jl:559-733 (gravity along -y) */
int kb_collide_boussinesq_3d(void *f, const void *Temp, const uint8_t *is_solid, int Nx, int Ny,
                             int Nz, double omega, double beta_g, double T_ref, int dtype,
                             void *stream);

/* fused_trt_libb_v2_step_3d!(f_out, f_in, rho, ux, uy, uz, is_solid, q_wall,
 *   uw_link_x, uw_link_y, uw_link_z, Nx, Ny, Nz, nu; Lambda)
 *   -- src/kernels/li_bb_3d_v2.jl:13-42 (bricks PullHalfwayBB_3D,
 * SolidInert_3D, ApplyLiBBPrePhase_3D, Moments_3D, CollideTRTDirect_3D,
 * WriteMoments_3D).  q_wall / uw_link_* are per-link arrays laid out like
 * f (19 planes, the population's type): q_wall > 0 marks a link cut by a
 * wall at that fraction of the link, uw_link_* the wall velocity there.
 * periodic as kb_fused_trt_step_3d.  KB_F64 / KB_F32. */
int kb_fused_trt_libb_step_3d(void *f_out, const void *f_in, void *rho, void *ux, void *uy,
                              void *uz, const uint8_t *is_solid, const void *q_wall,
                              const void *uw_link_x, const void *uw_link_y, const void *uw_link_z,
                              int Nx, int Ny, int Nz, double nu, double Lambda, int periodic,
                              int dtype, void *stream);

/* collide_guo_3d!(f, is_solid, omega, Fx, Fy, Fz) -- src/kernels/collide_guo_3d.jl:5-196 */
int kb_collide_guo_3d(void *f, const uint8_t *is_solid, int Nx, int Ny, int Nz, double omega,
                      double Fx, double Fy, double Fz, int dtype, void *stream);

/* collide_guo_field_3d!(f, is_solid, Fx_field, Fy_field, Fz_field, omega)
 *   -- src/kernels/collide_guo_3d.jl:199-332 */
int kb_collide_guo_field_3d(void *f, const uint8_t *is_solid, const void *Fx_field,
                            const void *Fy_field, const void *Fz_field, int Nx, int Ny, int Nz,
                            double omega, int dtype, void *stream);

/* Compact cut-link table (no counterpart in the reference; a B200 layout of
 * the inputs of fused_trt_libb_v2_step_3d!).  kb_libb_links_create gathers
 * the cut links of the dense arrays (q_wall, uw_link_x/y/z, dtype KB_F64 or
 * KB_F32, laid out like f) and the solid mask into one class byte per node
 * (fluid / solid / fluid with cut links) plus one record per node with cut
 * links, in node order.  It allocates the table, synchronises `stream` and
 * keeps no pointer to its inputs.  With the table, a step reads one byte per
 * node instead of the mask and 19 q_wall values. */
typedef struct kb_libb_links kb_libb_links;
int kb_libb_links_create(kb_libb_links **out, const uint8_t *is_solid, const void *q_wall,
                         const void *uw_link_x, const void *uw_link_y, const void *uw_link_z,
                         int Nx, int Ny, int Nz, int dtype, void *stream);
int kb_libb_links_destroy(kb_libb_links *links);
/* Number of nodes with cut links and the dtype of the stored link data. */
int kb_libb_links_info(const kb_libb_links *links, long long *nodes_with_links, int *dtype);

/* fused_trt_libb_v2_step_3d! with the compact table: KB_F64 / KB_F32
 * populations (table of the same dtype) give the same bits as
 * kb_fused_trt_libb_step_3d; the deviation storages (KB_F32 table) apply
 * the Bouzidi pre-phase to f - w and collide in FP32. */
int kb_fused_trt_libb_links_step_3d(void *f_out, const void *f_in, void *rho, void *ux, void *uy,
                                    void *uz, const kb_libb_links *links, double nu,
                                    double Lambda, int periodic, int dtype, void *stream);

/* Fused D3Q19 TRT step: the reference's 3D TRT kernel
 * fused_trt_libb_v2_step_3d!(f_out, f_in, rho, ux, uy, uz, is_solid, ...,
 * Nx, Ny, Nz, nu; Lambda) (src/kernels/li_bb_3d_v2.jl:31-42; bricks
 * PullHalfwayBB_3D, SolidInert_3D, Moments_3D, CollideTRTDirect_3D,
 * WriteMoments_3D in src/kernels/dsl/bricks_3d.jl:64-230, 476-483) with no
 * interpolated-wall link flagged.
 *   periodic: bit 0 = x, bit 1 = y, bit 2 = z wrap instead of half-way
 *             bounce-back (bit 2 alone = PullHalfwayBB_3D{true}).
 *   rho/ux/uy/uz: NULL skips the moment write (all four NULL or none).
 *   dtype: any kb_dtype.  KB_F64/KB_F32 follow the reference arithmetic;
 *   the *_DEV storages hold f - w_q and collide in FP32. */
int kb_fused_trt_step_3d(void *f_out, const void *f_in, void *rho, void *ux, void *uy, void *uz,
                         const uint8_t *is_solid, int Nx, int Ny, int Nz, double nu,
                         double Lambda, int periodic, int dtype, void *stream);

/* The same fused TRT step over the z-planes [k_begin, k_end) of an
 * allocation of Nz_alloc planes whose first and last planes are halo (ghost)
 * planes of a z-slab: z-pulls read planes k_begin - 1 and k_end as they are
 * (no wrap, no bounce-back).  All pointers address node (0, 0, 0) of the
 * whole allocation and every array spans it; only the planes of the range
 * are written.  Stepping [1, n) and [n, Nz_alloc - 1) gives bit for bit the
 * result of one step over [1, Nz_alloc - 1), so a slab steps its boundary
 * planes first, starts their exchange, then steps its interior.  Requires
 * 1 <= k_begin < k_end <= Nz_alloc - 1; periodic_xy: bit 0 = x, bit 1 = y.
 * No reference counterpart: the reference steps a whole array
 * (src/kernels/li_bb_3d_v2.jl:31). */
int kb_fused_trt_step_3d_zrange(void *f_out, const void *f_in, void *rho, void *ux, void *uy,
                                void *uz, const uint8_t *is_solid, int Nx, int Ny, int Nz_alloc,
                                int k_begin, int k_end, double nu, double Lambda,
                                int periodic_xy, int dtype, void *stream);

/* Kernel variant for tuning and tests (process-wide, not thread-safe to
 * change while other threads launch).  kernel 1 = the deviation-storage
 * kernels of kb_fused_trt_step_3d: 0 automatic (KB_F32_DEV: 3 for even Nx,
 * else 1; FP16/BF16: 5 when its conditions hold and the rows fill the
 * 256-node tiles to 90 % or more, else 2 when Nx >= 64, else 1), 1 one node
 * per thread, 2 nodes x and x+32 per thread, 3 adjacent node pairs with
 * 2-element vector accesses (even Nx), 4 adjacent node quads with 8-byte accesses
 * (16-bit storages, Nx % 4 == 0), 5 persistent row tiles of 256 nodes whose
 * pull source rows are staged in shared memory by tensor-memory-accelerator
 * copies (16-bit storages, Nx % 8 == 0, 16-byte aligned populations; two
 * rows per tile where Ny is even and the offsets fit in 32 bits), 6 the
 * staged kernel with one row per tile.  Variants 2 to 6 collide in packed
 * FP32x2 arithmetic.
 * kernel 2 = the tensor-core engine of the warm-start network and
 * kb_gemm_bf16: 0 warp-specialised persistent kernel with cp.async operand
 * staging, 1 one CTA per output tile with cp.async staging, 2 (default)
 * persistent kernel with tensor-memory-accelerator operand staging in
 * swizzled layouts (shapes it cannot tile run on engine 1).  Every variant
 * computes the same update up to FP32 rounding.  No reference counterpart. */
int kb_set_kernel_variant(int kernel, int variant);

/* stream_periodic_xz_movingwall_y_3d!(f_out, f_in, Ub, Ut, Nx, Ny, Nz; rho_w)
 *   -- src/kernels/stream_periodic_3d.jl:178 */
int kb_stream_periodic_xz_movingwall_y_3d(void *f_out, const void *f_in, double Ub, double Ut,
                                          double rho_w, int Nx, int Ny, int Nz, int dtype,
                                          void *stream);

/* --------------------------------------------- batched cavity sweeps -- */

/* Many lid-driven MRT cavities of different sizes in ONE persistent kernel:
 * the loop of test/test_mrt.jl:19-25 (stream_2d!, apply_zou_he_north_2d!,
 * collide_mrt_2d! with s_e = s_eps = 1.4, s_q = 1.2) per case, each run to
 * the steady residual r_u (src/drivers/gnf_periodic_steady.jl:186-194) or to
 * max_steps; a .krk Sweep (src/io/krk/parser.jl:362-420) maps to one batch.
 * Populations are stored as f - w_q in FP16/BF16/FP32 and collide in FP32.
 * No reference counterpart runs a sweep in one launch.  The handle owns its
 * device memory until kb_batch_destroy; creation synchronises `stream`. */
typedef struct kb_batch kb_batch;

int kb_batch_create(kb_batch **out, int n_cases, const int *N, const double *nu,
                    const double *u_lid, int dtype, void *stream);
int kb_batch_destroy(kb_batch *b);
/* Back to rest (f = w_q), all cases live; synchronises `stream`. */
int kb_batch_reset(kb_batch *b, void *stream);
/* Queue the run (asynchronous, one cooperative launch).  check_every >= 2;
 * max_steps a multiple of check_every; tile_nodes (multiple of 32) and
 * blocks_per_sm <= 0 take the autotuned choice (else 256 / occupancy). */
int kb_batch_run(kb_batch *b, int max_steps, int check_every, double tol, int tile_nodes,
                 int blocks_per_sm, void *stream);
/* Node updates done, live tiles left and the grid-barrier timeout flag
 * (KB_ERR_TIMEOUT if set); synchronises `stream`. */
int kb_batch_status(kb_batch *b, long long *updates, int *n_live, int *timed_out, void *stream);
/* Case c: size, steps run, last residual, state (0 live, 1 converged,
 * 2 hit max_steps, 3 non-finite) and optionally its final ux, uy (N*N floats,
 * row j = slow index); synchronises `stream`. */
int kb_batch_case(kb_batch *b, int c, int *N, int *steps, double *residual, int *state,
                  float *ux_host, float *uy_host, void *stream);
/* Time trial_steps of every (tile_nodes, blocks_per_sm) candidate (tiles of
 * 256 ... 4096 nodes, 1 ... the occupancy limit of blocks per SM), keep the
 * fastest for later runs; reports its MLUPS and that of the fixed schedule
 * kb_batch_run takes untuned (256-node tiles, as many blocks per SM as fit).
 * Resets the batch. */
int kb_batch_autotune(kb_batch *b, int trial_steps, int *best_tile, int *best_bpsm,
                      double *best_mlups, double *fixed_mlups, void *stream);
/* Device pointer to case c's final populations (9 planes of N*N, storage
 * `dtype`). */
int kb_batch_populations(kb_batch *b, int c, void **f, int *dtype, void *stream);

/* ---------------------------------------------------------- CUDA graphs -- */

/* Capture every library call issued on `stream` (a non-default stream)
 * between kb_graph_begin and kb_graph_end into an instantiated graph, then
 * replay it with kb_graph_launch.  This is the device-side form of
 * persistent_fused_bgk! / persistent_aa_bgk! (src/kernels/persistent_bgk_2d.jl:
 * 17-56), which queue Nt launches from the host.  Calls that synchronise or
 * allocate (kb_mass, kb_residual, kb_batch_create ...) cannot be captured. */
typedef struct kb_graph kb_graph;
int kb_graph_begin(void *stream);
int kb_graph_end(void *stream, kb_graph **out);
int kb_graph_launch(kb_graph *g, void *stream);
int kb_graph_destroy(kb_graph *g);

/* Self test of the bounded device wait used by the batched kernel's grid
 * barrier: one thread waits on a word that nothing changes; after `limit`
 * polls it gives up, sets the error flag and returns.  *timed_out = 1 and
 * KB_ERR_TIMEOUT is the expected result.  No reference counterpart. */
int kb_selftest_bounded_wait(long long limit, int *timed_out, void *stream);

/* ------------------------------------------------- precision utilities -- */

/* Convert populations between storages.  KB_*_DEV storages hold f - w_q; the
 * others hold f.  lattice_q is 9 (D2Q9) or 19 (D3Q19); n_nodes is the node
 * count of one population plane.  src and dst must not overlap.  No
 * reference counterpart (the reference stores plain f). */
int kb_convert_populations(void *dst, int dst_dtype, const void *src, int src_dtype,
                           int lattice_q, size_t n_nodes, void *stream);

/* Set the launch counter that seeds the random bits of the stochastic-rounding
 * storages on the current device (each launch that writes them advances it by
 * one).  Runs that start from the same populations and the same counter on
 * one stream are bit-identical.  Synchronises `stream`.  No reference
 * counterpart. */
int kb_set_stochastic_seed(unsigned int seed, void *stream);
/* The current value of that counter on the current device, so that a
 * checkpoint can record it and a resumed run can restore it with
 * kb_set_stochastic_seed and draw the same random bits as an uninterrupted
 * run.  Synchronises `stream`.  No reference counterpart. */
int kb_get_stochastic_seed(unsigned int *seed, void *stream);

/* *timed_out = 1 if a staged step (kernel 1, variant 5) gave up a bounded
 * wait on its copies since the last call (the flag is then cleared);
 * synchronises `stream`.  No reference counterpart. */
int kb_staged_step_status(int *timed_out, void *stream);

/* ---------------------------------------------------- FP64 reductions -- */

/* Total mass sum_q sum_nodes f (FP64, compensated), written to *out_host.
 * Synchronises `stream`.  Deviation storages add back w_q.  Returns
 * KB_ERR_NONFINITE (and still writes the sum) if any population is not
 * finite.  Replaces the host `sum(Array(rho))` of the reference drivers
 * (e.g. test/test_lbm_basic.jl:85-96). */
int kb_mass(const void *f, int lattice_q, size_t n_nodes, int dtype, double *out_host,
            void *stream);

/* kb_mass without any device allocation.  No counterpart in the reference:
 * it exists for callers that cannot let the library call cudaMalloc, such as
 * a host program whose own pool already owns the device memory, or a loop
 * that must not pay the device-wide synchronisation that cudaMalloc and
 * cudaFree bring.  The partial sums go to a fixed 256 KiB array in device
 * memory that the library holds on every GPU that loads it until the
 * process exits, so at most 1,073,479,680 populations (lattice_q * n_nodes)
 * fit; a larger call returns KB_ERR_ARG and names kb_mass.  The first call
 * on a device looks the array's address up (cudaGetSymbolAddress), so make
 * it before any stream capture; the address is kept for the life of the
 * process, so do not use this entry point on a device after
 * cudaDeviceReset.  All calls share the one array and each
 * call clears what must start at zero, but calls that overlap on the GPU
 * (other streams, other host threads) race.  Result, flag and
 * synchronisation as kb_mass. */
int kb_mass_static(const void *f, int lattice_q, size_t n_nodes, int dtype, double *out_host,
                   void *stream);

/* Steady residual r_u = ||u - u_prev||_2 / ||u||_2 over fluid nodes (FP64
 * accumulation), written to *out_host; synchronises `stream`.  uz/uz_prev
 * are NULL in 2D.  Fields are double for KB_F64, float otherwise.  The
 * definition is src/drivers/gnf_periodic_steady.jl:186-194. */
int kb_residual(const void *ux, const void *uy, const void *uz, const void *ux_prev,
                const void *uy_prev, const void *uz_prev, const uint8_t *is_solid,
                size_t n_nodes, int dtype, double *out_host, void *stream);

/* ------------------------------------------------ learned warm start -- */

/* The reference has no learned component.  These entry points add the warm
 * start: a 4-level convolutional encoder-decoder that maps a cavity's
 * (Re, N, wall mask) to its steady (rho, ux, uy).  Its forward, backward and
 * optimiser kernels are all in this library.  Every 3x3 convolution runs on
 * the BF16 tcgen05 tensor cores with FP32 accumulation in TMEM.  Activations
 * are NHWC BF16.  The first network channel of the input is 8. */

/* Plain GEMM on the same tensor-core mainloop: C[M][N] (FP32) = A B^T.  A is
 * [M][K] BF16 (a_mn = 0) or [K][M] (a_mn = 1); B is [N][K] (b_mn = 0) or
 * [K][N] (b_mn = 1).  M % 128 == 0, K % 64 == 0, N % 16 == 0.  *err_device
 * (device int) is set to 1 if a bounded wait inside the kernel gave up. */
int kb_gemm_bf16(const void *A, const void *B, float *C, int M, int N, int K, int a_mn,
                 int b_mn, int *err_device, void *stream);

typedef struct kb_surrogate kb_surrogate;
/* Network for inputs of H x W (multiples of 8) with `base_channels` (a
 * multiple of 16, 16..128) at the first level and batches of up to
 * `max_batch` cases.  Weights are He-normal from `seed`.  Allocates all its
 * device memory here; synchronises `stream`. */
int kb_surrogate_create(kb_surrogate **out, int max_batch, int H, int W, int base_channels,
                        unsigned long long seed, void *stream);
int kb_surrogate_destroy(kb_surrogate *s);
/* Number of FP32 parameters.  Layout: per layer W[cout][9*cin] (k = tap*cin +
 * c, tap = (dy+1)*3 + (dx+1)) then b[cout]; kb_surrogate_layer gives each
 * layer's offsets.  Layers: 0 enc1a, 1 enc1b, 2 enc2a, 3 enc2b, 4 enc3a,
 * 5 enc3b, 6 bott_a, 7 bott_b, 8 dec3a, 9 dec3b, 10 dec2a, 11 dec2b,
 * 12 dec1a, 13 dec1b, 14 head. */
int kb_surrogate_num_params(const kb_surrogate *s, long long *n);
int kb_surrogate_layer(const kb_surrogate *s, int layer, int *cin, int *cout, int *level,
                       long long *w_off, long long *b_off);
/* Output normalisation: the network predicts (x - offset) * scale for
 * x = (rho, ux, uy). */
int kb_surrogate_set_normalisation(kb_surrogate *s, const float *scale, const float *offset);
/* Weight gw of the gradient term of the training loss (default 0, the
 * mean-squared error): L = mean over pixels and channels of
 * e^2 + gw ((e(x+1) - e(x))^2 + (e(y+1) - e(y))^2), e = prediction - target. */
int kb_surrogate_set_grad_weight(kb_surrogate *s, float weight);
/* Copy the FP32 parameters out to `get` and/or in from `set` (device
 * pointers, n_params floats each); `set` also refreshes the BF16 copies. */
int kb_surrogate_params(kb_surrogate *s, float *get, const float *set, void *stream);
/* Copy the gradient of the last kb_surrogate_loss_backward to `get`. */
int kb_surrogate_grads(kb_surrogate *s, float *get, void *stream);
/* Build the NHWC BF16 input of n lid-driven cavities (device Re values). */
int kb_surrogate_cavity_inputs(const kb_surrogate *s, void *input, const float *re, int n,
                               int n_nodes, void *stream);
/* Forward pass; `out` (device, may be NULL) receives planar [n][3][H][W]
 * (rho, ux, uy) in physical units. */
int kb_surrogate_infer(kb_surrogate *s, const void *input, int n, float *out, void *stream);
/* Forward, mean-squared error against planar [n][3][H][W] targets, backward.
 * The loss (device float, may be NULL) and the parameter gradient are kept. */
int kb_surrogate_loss_backward(kb_surrogate *s, const void *input, const float *target, int n,
                               float *loss_out, void *stream);
/* One Adam update (bias-corrected, `step` counts from 1) with the last
 * gradient, then a refresh of the BF16 weight copies. */
int kb_surrogate_adam(kb_surrogate *s, float lr, float beta1, float beta2, float eps, int step,
                      void *stream);
/* kb_surrogate_loss_backward then kb_surrogate_adam (0.9, 0.999, 1e-8). */
int kb_surrogate_train_step(kb_surrogate *s, const void *input, const float *target, int n,
                            float lr, int step, float *loss_out, void *stream);
/* *timed_out = 1 if any tensor-core kernel of this network gave up a bounded
 * wait since creation; synchronises `stream`. */
int kb_surrogate_status(kb_surrogate *s, int *timed_out, void *stream);
/* Algorithmic FLOPs of one forward pass and of one training step for n cases. */
int kb_surrogate_flops(const kb_surrogate *s, int n, double *forward_flops, double *train_flops);

#ifdef __cplusplus
}
#endif

#endif /* KRAKENB200_H */
