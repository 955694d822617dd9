/*
 * kb_oracle.c -- CPU FP64 restatement of Kraken.jl's stream-collide path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle: the tests, the
 * smoke check and the CPU-baseline leg of the benchmark load it as a checker.
 * The product (the CUDA library behind include/krakenb200.h) never links,
 * calls or falls back to it.
 *
 * Every routine restates one Kraken.jl routine operation for operation: the
 * same left-to-right sums, `inv_rho = 1/rho` followed by a multiply, the same
 * pre-rounded constants (1/9, 1/36, ...), the same branch structure at the
 * domain edges.  It must be compiled with -ffp-contract=off so no multiply-add
 * is fused, which is what the reference's Julia CPU path does.  The citation
 * above each function names the reference file:line it follows.
 *
 * Parity pinning: Julia is not available in this environment, so the
 * reference cannot be run.  The restatement is pinned instead against the
 * known answers of the reference's own tests (lattice sums, TRT rates,
 * TRT == BGK, equilibrium stationarity, mass conservation, Ghia centreline,
 * Taylor-Green decay, half-way Dirichlet conduction, De Vahl Davis Nu); see
 * tests/test_oracle_pins.py.
 *
 * Layout: Julia column-major arrays, 0-based here.
 *   2D  f[i + Nx*(j + Ny*q)]            (i fastest, then j, then population q)
 *   3D  f[i + Nx*(j + Ny*(k + Nz*q))]
 * Population q is 0-based here; the reference's q is 1-based (q_ref = q + 1).
 * Masks are one byte per node (Julia Bool).
 */
#include <math.h>
#include <stdint.h>
#include <stddef.h>
#include <string.h>
#include <stdlib.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define I2(i, j, q) ((size_t)(i) + (size_t)Nx * ((size_t)(j) + (size_t)Ny * (size_t)(q)))
#define N2(i, j) ((size_t)(i) + (size_t)Nx * (size_t)(j))
#define I3(i, j, k, q) \
    ((size_t)(i) + (size_t)Nx * ((size_t)(j) + (size_t)Ny * ((size_t)(k) + (size_t)Nz * (size_t)(q))))
#define N3(i, j, k) ((size_t)(i) + (size_t)Nx * ((size_t)(j) + (size_t)Ny * (size_t)(k)))

/* ------------------------------------------------------------------------ */
/* Lattice constants: src/lattice/d2q9.jl:17-29, src/lattice/d3q19.jl:13-47  */
/* ------------------------------------------------------------------------ */
const double or_d2q9_w[9] = {4.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0,
                             1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0};
const int or_d2q9_cx[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
const int or_d2q9_cy[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
const int or_d2q9_opp[9] = {0, 3, 4, 1, 2, 7, 8, 5, 6};

const double or_d3q19_w[19] = {1.0 / 3.0,
                               1.0 / 18.0, 1.0 / 18.0, 1.0 / 18.0, 1.0 / 18.0, 1.0 / 18.0, 1.0 / 18.0,
                               1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0,
                               1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0,
                               1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0};
const int or_d3q19_cx[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
const int or_d3q19_cy[19] = {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1};
const int or_d3q19_cz[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1};
const int or_d3q19_opp[19] = {0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15};

void or_lattice_d2q9(double *w, int *cx, int *cy, int *opp) {
    for (int q = 0; q < 9; ++q) {
        w[q] = or_d2q9_w[q]; cx[q] = or_d2q9_cx[q]; cy[q] = or_d2q9_cy[q]; opp[q] = or_d2q9_opp[q];
    }
}

void or_lattice_d3q19(double *w, int *cx, int *cy, int *cz, int *opp) {
    for (int q = 0; q < 19; ++q) {
        w[q] = or_d3q19_w[q]; cx[q] = or_d3q19_cx[q]; cy[q] = or_d3q19_cy[q];
        cz[q] = or_d3q19_cz[q]; opp[q] = or_d3q19_opp[q];
    }
}

/* equilibrium(::D2Q9, rho, ux, uy, q): src/lattice/d2q9.jl:60-67 */
double or_equilibrium_d2q9(double rho, double ux, double uy, int q) {
    double w = or_d2q9_w[q];
    double cx = (double)or_d2q9_cx[q], cy = (double)or_d2q9_cy[q];
    double cu = cx * ux + cy * uy;
    double usq = ux * ux + uy * uy;
    return w * rho * (1.0 + 3.0 * cu + 4.5 * cu * cu - 1.5 * usq);
}

/* equilibrium(::D3Q19, rho, ux, uy, uz, q): src/lattice/d3q19.jl:67-75 */
double or_equilibrium_d3q19(double rho, double ux, double uy, double uz, int q) {
    double w = or_d3q19_w[q];
    double cx = (double)or_d3q19_cx[q], cy = (double)or_d3q19_cy[q], cz = (double)or_d3q19_cz[q];
    double cu = cx * ux + cy * uy + cz * uz;
    double usq = ux * ux + uy * uy + uz * uz;
    return w * rho * (1.0 + 3.0 * cu + 4.5 * cu * cu - 1.5 * usq);
}

/* ------------------------------------------------------------------------ */
/* feq_2d / moments_2d: src/kernels/equilibrium_helpers.jl:8-61             */
/* ------------------------------------------------------------------------ */
static inline double feq_poly(double w, double rho, double cu, double usq) {
    return w * rho * (1.0 + 3.0 * cu + 4.5 * cu * cu - 1.5 * usq);
}

static inline void feq2d_all(double rho, double ux, double uy, double usq, double *feq) {
    feq[0] = 4.0 / 9.0 * rho * (1.0 - 1.5 * usq);
    feq[1] = feq_poly(1.0 / 9.0, rho, ux, usq);
    feq[2] = feq_poly(1.0 / 9.0, rho, uy, usq);
    feq[3] = feq_poly(1.0 / 9.0, rho, -ux, usq);
    feq[4] = feq_poly(1.0 / 9.0, rho, -uy, usq);
    feq[5] = feq_poly(1.0 / 36.0, rho, ux + uy, usq);
    feq[6] = feq_poly(1.0 / 36.0, rho, -ux + uy, usq);
    feq[7] = feq_poly(1.0 / 36.0, rho, -ux - uy, usq);
    feq[8] = feq_poly(1.0 / 36.0, rho, ux - uy, usq);
}

static inline void moments2d(const double *p, double *rho, double *ux, double *uy) {
    double r = p[0] + p[1] + p[2] + p[3] + p[4] + p[5] + p[6] + p[7] + p[8];
    double inv = 1.0 / r;
    *rho = r;
    *ux = (p[1] - p[3] + p[5] - p[6] - p[7] + p[8]) * inv;
    *uy = (p[2] - p[4] + p[5] + p[6] - p[7] - p[8]) * inv;
}

/* Pull with half-way bounce-back on all four edges.
 * src/kernels/collide_stream_2d.jl:12-23 (identical in fused_bgk_2d.jl:13-24,
 * fused_trt_2d.jl:39-51, aa_bgk_2d.jl:17-29, fused_thermal_2d.jl:10-25). */
static inline void pull2d(const double *f, int Nx, int Ny, int i, int j, double *fp) {
    int im = i > 0 ? i - 1 : 0, ip = i < Nx - 1 ? i + 1 : Nx - 1;
    int jm = j > 0 ? j - 1 : 0, jp = j < Ny - 1 ? j + 1 : Ny - 1;
    fp[0] = f[I2(i, j, 0)];
    fp[1] = (i > 0) ? f[I2(im, j, 1)] : f[I2(i, j, 3)];
    fp[2] = (j > 0) ? f[I2(i, jm, 2)] : f[I2(i, j, 4)];
    fp[3] = (i < Nx - 1) ? f[I2(ip, j, 3)] : f[I2(i, j, 1)];
    fp[4] = (j < Ny - 1) ? f[I2(i, jp, 4)] : f[I2(i, j, 2)];
    fp[5] = (i > 0 && j > 0) ? f[I2(im, jm, 5)] : f[I2(i, j, 7)];
    fp[6] = (i < Nx - 1 && j > 0) ? f[I2(ip, jm, 6)] : f[I2(i, j, 8)];
    fp[7] = (i < Nx - 1 && j < Ny - 1) ? f[I2(ip, jp, 7)] : f[I2(i, j, 5)];
    fp[8] = (i > 0 && j < Ny - 1) ? f[I2(im, jp, 8)] : f[I2(i, j, 6)];
}

/* stream_2d!: src/kernels/collide_stream_2d.jl:5-31, 77-82 */
void or_stream_2d(double *f_out, const double *f_in, int Nx, int Ny) {
#pragma omp parallel for schedule(static)
    for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i) {
            double fp[9];
            pull2d(f_in, Nx, Ny, i, j, fp);
            for (int q = 0; q < 9; ++q) f_out[I2(i, j, q)] = fp[q];
        }
}

/* bounce_back_2d!: src/kernels/equilibrium_helpers.jl:65-70 */
static inline void swap_pairs_2d(double *p) {
    double t;
    t = p[1]; p[1] = p[3]; p[3] = t;
    t = p[2]; p[2] = p[4]; p[4] = t;
    t = p[5]; p[5] = p[7]; p[7] = t;
    t = p[6]; p[6] = p[8]; p[8] = t;
}

/* collide_2d!: src/kernels/collide_stream_2d.jl:35-61, 96-102 */
void or_collide_2d(double *f, const uint8_t *solid, int Nx, int Ny, double omega) {
#pragma omp parallel for schedule(static)
    for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i) {
            double p[9];
            for (int q = 0; q < 9; ++q) p[q] = f[I2(i, j, q)];
            if (solid && solid[N2(i, j)]) {
                swap_pairs_2d(p);
            } else {
                double rho, ux, uy, feq[9];
                moments2d(p, &rho, &ux, &uy);
                double usq = ux * ux + uy * uy;
                feq2d_all(rho, ux, uy, usq, feq);
                for (int q = 0; q < 9; ++q) p[q] = p[q] - omega * (p[q] - feq[q]);
            }
            for (int q = 0; q < 9; ++q) f[I2(i, j, q)] = p[q];
        }
}

/* apply_zou_he_north_2d!: src/kernels/boundary_2d.jl:13-60 */
void or_zou_he_north_2d(double *f, double u, int Nx, int Ny) {
    int j = Ny - 1;
    for (int i = 0; i < Nx; ++i) {
        double f1 = f[I2(i, j, 0)], f2 = f[I2(i, j, 1)], f3 = f[I2(i, j, 2)];
        double f4 = f[I2(i, j, 3)], f6 = f[I2(i, j, 5)], f7 = f[I2(i, j, 6)];
        double rw = (f1 + f2 + f4 + 2.0 * (f3 + f6 + f7)) / (1.0 + u * 0.0);
        f[I2(i, j, 4)] = f3;
        f[I2(i, j, 8)] = f7 - 0.5 * (f2 - f4) + 0.5 * rw * u;
        f[I2(i, j, 7)] = f6 + 0.5 * (f2 - f4) - 0.5 * rw * u;
    }
}

/* apply_zou_he_south_2d!: src/kernels/boundary_2d.jl:135-167 */
void or_zou_he_south_2d(double *f, double u, int Nx, int Ny) {
    int j = 0;
    for (int i = 0; i < Nx; ++i) {
        double f1 = f[I2(i, j, 0)], f2 = f[I2(i, j, 1)], f4 = f[I2(i, j, 3)];
        double f5 = f[I2(i, j, 4)], f8 = f[I2(i, j, 7)], f9 = f[I2(i, j, 8)];
        double rw = f1 + f2 + f4 + 2.0 * (f5 + f8 + f9);
        f[I2(i, j, 2)] = f5;
        f[I2(i, j, 5)] = f8 - 0.5 * (f2 - f4) + 0.5 * rw * u;
        f[I2(i, j, 6)] = f9 + 0.5 * (f2 - f4) - 0.5 * rw * u;
    }
}

/* apply_zou_he_west_2d!: src/kernels/boundary_2d.jl:171-202 */
void or_zou_he_west_2d(double *f, double u_in, int Nx, int Ny) {
    for (int j = 0; j < Ny; ++j) {
        double f1 = f[I2(0, j, 0)], f3 = f[I2(0, j, 2)], f4 = f[I2(0, j, 3)];
        double f5 = f[I2(0, j, 4)], f7 = f[I2(0, j, 6)], f8 = f[I2(0, j, 7)];
        double rw = (f1 + f3 + f5 + 2.0 * (f4 + f7 + f8)) / (1.0 - u_in);
        f[I2(0, j, 1)] = f4 + 2.0 / 3.0 * rw * u_in;
        f[I2(0, j, 5)] = f8 - 0.5 * (f3 - f5) + 1.0 / 6.0 * rw * u_in;
        f[I2(0, j, 8)] = f7 + 0.5 * (f3 - f5) + 1.0 / 6.0 * rw * u_in;
    }
}

/* apply_zou_he_pressure_east_2d!: src/kernels/boundary_2d.jl:206-241 */
void or_zou_he_pressure_east_2d(double *f, int Nx, int Ny, double rho_out) {
    int i = Nx - 1;
    for (int j = 0; j < Ny; ++j) {
        double f1 = f[I2(i, j, 0)], f2 = f[I2(i, j, 1)], f3 = f[I2(i, j, 2)];
        double f5 = f[I2(i, j, 4)], f6 = f[I2(i, j, 5)], f9 = f[I2(i, j, 8)];
        double ux = -1.0 + (f1 + f3 + f5 + 2.0 * (f2 + f6 + f9)) / rho_out;
        f[I2(i, j, 3)] = f2 - 2.0 / 3.0 * rho_out * ux;
        f[I2(i, j, 6)] = f9 - 0.5 * (f3 - f5) - 1.0 / 6.0 * rho_out * ux;
        f[I2(i, j, 7)] = f6 + 0.5 * (f3 - f5) - 1.0 / 6.0 * rho_out * ux;
    }
}

/* apply_zou_he_pressure_west_2d!: src/kernels/boundary_2d.jl:264-299 */
void or_zou_he_pressure_west_2d(double *f, int Nx, int Ny, double rho_in) {
    (void)Nx;
    for (int j = 0; j < Ny; ++j) {
        double f1 = f[I2(0, j, 0)], f3 = f[I2(0, j, 2)], f4 = f[I2(0, j, 3)];
        double f5 = f[I2(0, j, 4)], f7 = f[I2(0, j, 6)], f8 = f[I2(0, j, 7)];
        double ux = 1.0 - (f1 + f3 + f5 + 2.0 * (f4 + f7 + f8)) / rho_in;
        f[I2(0, j, 1)] = f4 + 2.0 / 3.0 * rho_in * ux;
        f[I2(0, j, 5)] = f8 - 0.5 * (f3 - f5) + 1.0 / 6.0 * rho_in * ux;
        f[I2(0, j, 8)] = f7 + 0.5 * (f3 - f5) + 1.0 / 6.0 * rho_in * ux;
    }
}

/* apply_extrapolate_east_2d!: src/kernels/boundary_2d.jl:303-323 */
void or_extrapolate_east_2d(double *f, int Nx, int Ny) {
    for (int j = 0; j < Ny; ++j)
        for (int q = 0; q < 9; ++q) f[I2(Nx - 1, j, q)] = f[I2(Nx - 2, j, q)];
}

/* bounce_back_walls_2d_kernel!: src/kernels/boundary_2d.jl:64-90.
 * wall_id: 1 south, 2 west, 3 east, 4 north (same codes as the reference). */
void or_bounce_back_wall_2d(double *f, int Nx, int Ny, int wall_id) {
    if (wall_id == 1) {
        for (int i = 0; i < Nx; ++i) {
            f[I2(i, 0, 2)] = f[I2(i, 0, 4)];
            f[I2(i, 0, 5)] = f[I2(i, 0, 7)];
            f[I2(i, 0, 6)] = f[I2(i, 0, 8)];
        }
    } else if (wall_id == 2) {
        for (int j = 0; j < Ny; ++j) {
            f[I2(0, j, 1)] = f[I2(0, j, 3)];
            f[I2(0, j, 5)] = f[I2(0, j, 7)];
            f[I2(0, j, 8)] = f[I2(0, j, 6)];
        }
    } else if (wall_id == 3) {
        for (int j = 0; j < Ny; ++j) {
            f[I2(Nx - 1, j, 3)] = f[I2(Nx - 1, j, 1)];
            f[I2(Nx - 1, j, 6)] = f[I2(Nx - 1, j, 8)];
            f[I2(Nx - 1, j, 7)] = f[I2(Nx - 1, j, 5)];
        }
    } else if (wall_id == 4) {
        for (int i = 0; i < Nx; ++i) {
            f[I2(i, Ny - 1, 4)] = f[I2(i, Ny - 1, 2)];
            f[I2(i, Ny - 1, 7)] = f[I2(i, Ny - 1, 5)];
            f[I2(i, Ny - 1, 8)] = f[I2(i, Ny - 1, 6)];
        }
    }
}

/* compute_macroscopic_2d!: src/kernels/macroscopic.jl:5-38 */
void or_macroscopic_2d(double *rho, double *ux, double *uy, const double *f, int Nx, int Ny) {
#pragma omp parallel for schedule(static)
    for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i) {
            double p[9];
            for (int q = 0; q < 9; ++q) p[q] = f[I2(i, j, q)];
            double r = p[0] + p[1] + p[2] + p[3] + p[4] + p[5] + p[6] + p[7] + p[8];
            double inv = 1.0 / r;
            rho[N2(i, j)] = r;
            ux[N2(i, j)] = (p[1] - p[3] + p[5] - p[6] - p[7] + p[8]) * inv;
            uy[N2(i, j)] = (p[2] - p[4] + p[5] + p[6] - p[7] - p[8]) * inv;
        }
}

/* fused_bgk_step!: src/kernels/fused_bgk_2d.jl:8-72 */
void or_fused_bgk_2d(double *f_out, const double *f_in, double *rho_o, double *ux_o, double *uy_o,
                     const uint8_t *solid, int Nx, int Ny, double omega) {
#pragma omp parallel for schedule(static)
    for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i) {
            double p[9];
            pull2d(f_in, Nx, Ny, i, j, p);
            if (solid && solid[N2(i, j)]) {
                swap_pairs_2d(p);
                for (int q = 0; q < 9; ++q) f_out[I2(i, j, q)] = p[q];
                rho_o[N2(i, j)] = 1.0; ux_o[N2(i, j)] = 0.0; uy_o[N2(i, j)] = 0.0;
            } else {
                double rho, ux, uy, feq[9];
                moments2d(p, &rho, &ux, &uy);
                double usq = ux * ux + uy * uy;
                feq2d_all(rho, ux, uy, usq, feq);
                for (int q = 0; q < 9; ++q) f_out[I2(i, j, q)] = p[q] - omega * (p[q] - feq[q]);
                rho_o[N2(i, j)] = rho; ux_o[N2(i, j)] = ux; uy_o[N2(i, j)] = uy;
            }
        }
}

/* Lid-driven cavity with a moving-wall half-way bounce-back lid: the DSL
 * composition PullHalfwayBB -> ApplyHalfwayBBPrePhase -> Moments ->
 * CollideBGK -> WriteMoments (src/kernels/dsl/bricks.jl:447-487 for the lid
 * link rule; the pull and BGK as fused_bgk_2d.jl:8-59).  The top row's three
 * north-pointing links (q = 3, 6, 7 in the reference's 1-based numbering) are
 * cut by a wall moving at (u_lid, 0), corners included:
 *   fp5 = f_in[3] - (2/3)*0,  fp8 = f_in[6] - (1/6)(u_lid + 0),
 *   fp9 = f_in[7] - (1/6)(-u_lid + 0). */
static inline void lid_links(const double *f, int Nx, int Ny, int i, int j, double u, double *fp) {
    if (j != Ny - 1) return;
    const double d5 = -(2.0 / 3.0) * 0.0;
    const double d8 = -(1.0 / 6.0) * (u + 0.0);
    const double d9 = -(1.0 / 6.0) * (-u + 0.0);
    fp[4] = f[I2(i, j, 2)] + d5;
    fp[7] = f[I2(i, j, 5)] + d8;
    fp[8] = f[I2(i, j, 6)] + d9;
}

void or_cavity_movingwall_bgk_2d(double *f_out, const double *f_in, double *rho_o, double *ux_o,
                                 double *uy_o, const uint8_t *solid, int Nx, int Ny, double omega,
                                 double u_lid) {
#pragma omp parallel for schedule(static)
    for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i) {
            double p[9];
            pull2d(f_in, Nx, Ny, i, j, p);
            if (solid && solid[N2(i, j)]) {
                swap_pairs_2d(p);
                for (int q = 0; q < 9; ++q) f_out[I2(i, j, q)] = p[q];
                rho_o[N2(i, j)] = 1.0; ux_o[N2(i, j)] = 0.0; uy_o[N2(i, j)] = 0.0;
                continue;
            }
            lid_links(f_in, Nx, Ny, i, j, u_lid, p);
            double rho, ux, uy, feq[9];
            moments2d(p, &rho, &ux, &uy);
            double usq = ux * ux + uy * uy;
            feq2d_all(rho, ux, uy, usq, feq);
            for (int q = 0; q < 9; ++q) f_out[I2(i, j, q)] = p[q] - omega * (p[q] - feq[q]);
            rho_o[N2(i, j)] = rho; ux_o[N2(i, j)] = ux; uy_o[N2(i, j)] = uy;
        }
}

/* trt_rates(nu; Lambda): src/kernels/fused_trt_2d.jl:129-133 */
void or_trt_rates(double nu, double lambda, double *s_plus, double *s_minus) {
    *s_plus = 1.0 / (3.0 * nu + 0.5);
    *s_minus = 1.0 / (lambda / (3.0 * nu) + 0.5);
}

/* TRT collide of one node given pulled p[] (fused_trt_2d.jl:65-94). */
static inline void trt2d_node(double *p, double sp, double sm, double *rho, double *ux, double *uy) {
    double feq[9];
    moments2d(p, rho, ux, uy);
    double usq = (*ux) * (*ux) + (*uy) * (*uy);
    feq2d_all(*rho, *ux, *uy, usq, feq);
    double a = (sp + sm) * 0.5, b = (sp - sm) * 0.5;
    double o[9];
    o[0] = p[0] - sp * (p[0] - feq[0]);
    o[1] = p[1] - a * (p[1] - feq[1]) - b * (p[3] - feq[3]);
    o[3] = p[3] - a * (p[3] - feq[3]) - b * (p[1] - feq[1]);
    o[2] = p[2] - a * (p[2] - feq[2]) - b * (p[4] - feq[4]);
    o[4] = p[4] - a * (p[4] - feq[4]) - b * (p[2] - feq[2]);
    o[5] = p[5] - a * (p[5] - feq[5]) - b * (p[7] - feq[7]);
    o[7] = p[7] - a * (p[7] - feq[7]) - b * (p[5] - feq[5]);
    o[6] = p[6] - a * (p[6] - feq[6]) - b * (p[8] - feq[8]);
    o[8] = p[8] - a * (p[8] - feq[8]) - b * (p[6] - feq[6]);
    for (int q = 0; q < 9; ++q) p[q] = o[q];
}

/* fused_trt_step!: src/kernels/fused_trt_2d.jl:29-101, 145-153.  The caller
 * passes the rates already rounded to the storage type (as ET(s_plus)). */
void or_fused_trt_2d(double *f_out, const double *f_in, double *rho_o, double *ux_o, double *uy_o,
                     const uint8_t *solid, int Nx, int Ny, double sp, double sm) {
#pragma omp parallel for schedule(static)
    for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i) {
            double p[9];
            pull2d(f_in, Nx, Ny, i, j, p);
            if (solid && solid[N2(i, j)]) {
                swap_pairs_2d(p);
                for (int q = 0; q < 9; ++q) f_out[I2(i, j, q)] = p[q];
                rho_o[N2(i, j)] = 1.0; ux_o[N2(i, j)] = 0.0; uy_o[N2(i, j)] = 0.0;
            } else {
                double rho, ux, uy;
                trt2d_node(p, sp, sm, &rho, &ux, &uy);
                for (int q = 0; q < 9; ++q) f_out[I2(i, j, q)] = p[q];
                rho_o[N2(i, j)] = rho; ux_o[N2(i, j)] = ux; uy_o[N2(i, j)] = uy;
            }
        }
}

/* collide_mrt_2d!: src/kernels/collide_mrt_2d.jl:43-125.  s_nu is passed in
 * already computed as 1/(3 nu + 0.5) (collide_mrt_2d.jl:122). */
void or_collide_mrt_2d(double *f, const uint8_t *solid, int Nx, int Ny,
                       double s_e, double s_eps, double s_q, double s_nu) {
#pragma omp parallel for schedule(static)
    for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i) {
            double p[9];
            for (int q = 0; q < 9; ++q) p[q] = f[I2(i, j, q)];
            if (solid && solid[N2(i, j)]) {
                swap_pairs_2d(p);
                for (int q = 0; q < 9; ++q) f[I2(i, j, q)] = p[q];
                continue;
            }
            double f1 = p[0], f2 = p[1], f3 = p[2], f4 = p[3], f5 = p[4];
            double f6 = p[5], f7 = p[6], f8 = p[7], f9 = p[8];
            double rho = f1 + f2 + f3 + f4 + f5 + f6 + f7 + f8 + f9;
            double e = -4.0 * f1 - f2 - f3 - f4 - f5 + 2.0 * (f6 + f7 + f8 + f9);
            double eps = 4.0 * f1 - 2.0 * (f2 + f3 + f4 + f5) + f6 + f7 + f8 + f9;
            double jx = f2 - f4 + f6 - f7 - f8 + f9;
            double qx = -2.0 * f2 + 2.0 * f4 + f6 - f7 - f8 + f9;
            double jy = f3 - f5 + f6 + f7 - f8 - f9;
            double qy = -2.0 * f3 + 2.0 * f5 + f6 + f7 - f8 - f9;
            double pxx = f2 - f3 + f4 - f5;
            double pxy = f6 - f7 + f8 - f9;
            double inv = 1.0 / rho;
            double ux = jx * inv, uy = jy * inv;
            double usq = ux * ux + uy * uy;
            double e_eq = -2.0 * rho + 3.0 * rho * usq;
            double eps_eq = rho - 3.0 * rho * usq;
            double qx_eq = -rho * ux;
            double qy_eq = -rho * uy;
            double pxx_eq = rho * (ux * ux - uy * uy);
            double pxy_eq = rho * ux * uy;
            double es = e - s_e * (e - e_eq);
            double ep = eps - s_eps * (eps - eps_eq);
            double qxs = qx - s_q * (qx - qx_eq);
            double qys = qy - s_q * (qy - qy_eq);
            double ps = pxx - s_nu * (pxx - pxx_eq);
            double pxys = pxy - s_nu * (pxy - pxy_eq);
            double r = rho, jxs = jx, jys = jy;
            const double c9 = 1.0 / 9.0, c36 = 1.0 / 36.0, c18 = 1.0 / 18.0, c6 = 1.0 / 6.0,
                         c4 = 1.0 / 4.0, c12 = 1.0 / 12.0;
            f[I2(i, j, 0)] = c9 * r - c9 * es + c9 * ep;
            f[I2(i, j, 1)] = c9 * r - c36 * es - c18 * ep + c6 * jxs - c6 * qxs + c4 * ps;
            f[I2(i, j, 2)] = c9 * r - c36 * es - c18 * ep + c6 * jys - c6 * qys - c4 * ps;
            f[I2(i, j, 3)] = c9 * r - c36 * es - c18 * ep - c6 * jxs + c6 * qxs + c4 * ps;
            f[I2(i, j, 4)] = c9 * r - c36 * es - c18 * ep - c6 * jys + c6 * qys - c4 * ps;
            f[I2(i, j, 5)] = c9 * r + c18 * es + c36 * ep + c6 * jxs + c12 * qxs + c6 * jys + c12 * qys + c4 * pxys;
            f[I2(i, j, 6)] = c9 * r + c18 * es + c36 * ep - c6 * jxs - c12 * qxs + c6 * jys + c12 * qys - c4 * pxys;
            f[I2(i, j, 7)] = c9 * r + c18 * es + c36 * ep - c6 * jxs - c12 * qxs - c6 * jys - c12 * qys + c4 * pxys;
            f[I2(i, j, 8)] = c9 * r + c18 * es + c36 * ep + c6 * jxs + c12 * qxs - c6 * jys - c12 * qys - c4 * pxys;
        }
}

/* stream_fully_periodic_2d!: src/kernels/stream_periodic_2d.jl:79-117 */
void or_stream_fully_periodic_2d(double *f_out, const double *f_in, int Nx, int Ny) {
#pragma omp parallel for schedule(static)
    for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i) {
            int ip = i > 0 ? i - 1 : Nx - 1, im = i < Nx - 1 ? i + 1 : 0;
            int jp = j > 0 ? j - 1 : Ny - 1, jm = j < Ny - 1 ? j + 1 : 0;
            f_out[I2(i, j, 0)] = f_in[I2(i, j, 0)];
            f_out[I2(i, j, 1)] = f_in[I2(ip, j, 1)];
            f_out[I2(i, j, 2)] = f_in[I2(i, jp, 2)];
            f_out[I2(i, j, 3)] = f_in[I2(im, j, 3)];
            f_out[I2(i, j, 4)] = f_in[I2(i, jm, 4)];
            f_out[I2(i, j, 5)] = f_in[I2(ip, jp, 5)];
            f_out[I2(i, j, 6)] = f_in[I2(im, jp, 6)];
            f_out[I2(i, j, 7)] = f_in[I2(im, jm, 7)];
            f_out[I2(i, j, 8)] = f_in[I2(ip, jm, 8)];
        }
}

/* stream_periodic_x_wall_y_2d!: src/kernels/stream_periodic_2d.jl:5-75 */
void or_stream_periodic_x_wall_y_2d(double *f_out, const double *f_in, int Nx, int Ny) {
#pragma omp parallel for schedule(static)
    for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i) {
            int jm1 = j > 0 ? j - 1 : j, jp1 = j < Ny - 1 ? j + 1 : j;
            int iw = i > 0 ? i - 1 : Nx - 1, ie = i < Nx - 1 ? i + 1 : 0;
            f_out[I2(i, j, 0)] = f_in[I2(i, j, 0)];
            f_out[I2(i, j, 1)] = f_in[I2(iw, j, 1)];
            f_out[I2(i, j, 2)] = j > 0 ? f_in[I2(i, jm1, 2)] : f_in[I2(i, j, 4)];
            f_out[I2(i, j, 3)] = f_in[I2(ie, j, 3)];
            f_out[I2(i, j, 4)] = j < Ny - 1 ? f_in[I2(i, jp1, 4)] : f_in[I2(i, j, 2)];
            f_out[I2(i, j, 5)] = j > 0 ? f_in[I2(iw, jm1, 5)] : f_in[I2(i, j, 7)];
            f_out[I2(i, j, 6)] = j > 0 ? f_in[I2(ie, jm1, 6)] : f_in[I2(i, j, 8)];
            f_out[I2(i, j, 7)] = j < Ny - 1 ? f_in[I2(ie, jp1, 7)] : f_in[I2(i, j, 5)];
            f_out[I2(i, j, 8)] = j < Ny - 1 ? f_in[I2(iw, jp1, 8)] : f_in[I2(i, j, 6)];
        }
}

/* The path-B cavity driver, run_cavity_2d: src/drivers/basic.jl:112-144.
 * f_in/f_out ping-pong; on return f_a holds the latest populations. */
void or_run_cavity_2d(double *f_a, double *f_b, double *rho, double *ux, double *uy,
                      const uint8_t *solid, int Nx, int Ny, double omega, double u_lid, int steps) {
    double *fi = f_a, *fo = f_b;
    size_t n = (size_t)Nx * Ny * 9;
    for (int s = 0; s < steps; ++s) {
        or_stream_2d(fo, fi, Nx, Ny);
        or_zou_he_north_2d(fo, u_lid, Nx, Ny);
        or_collide_2d(fo, solid, Nx, Ny, omega);
        or_macroscopic_2d(rho, ux, uy, fo, Nx, Ny);
        double *t = fi; fi = fo; fo = t;
    }
    if (fi != f_a) memcpy(f_a, fi, n * sizeof(double));
}

/* ------------------------------------------------------------------------ */
/* D3Q19                                                                     */
/* ------------------------------------------------------------------------ */

static inline void feq3d_all(double rho, double ux, double uy, double uz, double usq, double *feq) {
    const double wr = 1.0 / 3.0, wa = 1.0 / 18.0, we = 1.0 / 36.0;
    feq[0] = wr * rho * (1.0 - 1.5 * usq);
    feq[1] = feq_poly(wa, rho, ux, usq);
    feq[2] = feq_poly(wa, rho, -ux, usq);
    feq[3] = feq_poly(wa, rho, uy, usq);
    feq[4] = feq_poly(wa, rho, -uy, usq);
    feq[5] = feq_poly(wa, rho, uz, usq);
    feq[6] = feq_poly(wa, rho, -uz, usq);
    feq[7] = feq_poly(we, rho, ux + uy, usq);
    feq[8] = feq_poly(we, rho, -ux + uy, usq);
    feq[9] = feq_poly(we, rho, ux - uy, usq);
    feq[10] = feq_poly(we, rho, -ux - uy, usq);
    feq[11] = feq_poly(we, rho, ux + uz, usq);
    feq[12] = feq_poly(we, rho, -ux + uz, usq);
    feq[13] = feq_poly(we, rho, ux - uz, usq);
    feq[14] = feq_poly(we, rho, -ux - uz, usq);
    feq[15] = feq_poly(we, rho, uy + uz, usq);
    feq[16] = feq_poly(we, rho, -uy + uz, usq);
    feq[17] = feq_poly(we, rho, uy - uz, usq);
    feq[18] = feq_poly(we, rho, -uy - uz, usq);
}

/* moments_3d: src/kernels/equilibrium_helpers_3d.jl:102-112 (also
 * collide_stream_3d.jl:69-73 and macroscopic.jl:53-59, same order). */
static inline void moments3d(const double *p, double *rho, double *ux, double *uy, double *uz) {
    double r = p[0] + p[1] + p[2] + p[3] + p[4] + p[5] + p[6] + p[7] + p[8] + p[9] +
               p[10] + p[11] + p[12] + p[13] + p[14] + p[15] + p[16] + p[17] + p[18];
    double inv = 1.0 / r;
    *rho = r;
    *ux = (p[1] - p[2] + p[7] - p[8] + p[9] - p[10] + p[11] - p[12] + p[13] - p[14]) * inv;
    *uy = (p[3] - p[4] + p[7] + p[8] - p[9] - p[10] + p[15] - p[16] + p[17] - p[18]) * inv;
    *uz = (p[5] - p[6] + p[11] + p[12] - p[13] - p[14] + p[15] + p[16] - p[17] - p[18]) * inv;
}

/* Pull with half-way bounce-back, per-axis optionally periodic.
 * Walls on every axis: src/kernels/collide_stream_3d.jl:5-42 and the DSL brick
 * PullHalfwayBB_3D{false} (src/kernels/dsl/bricks_3d.jl:70-100).  Periodic z:
 * PullHalfwayBB_3D{true} (bricks_3d.jl:106-136).  Periodic x and y are the
 * same wrap rule extended to the other two axes (no reference counterpart; the
 * reference has no fully periodic D3Q19 pull). */
static inline void pull3d(const double *f, int Nx, int Ny, int Nz, int i, int j, int k,
                          int per_x, int per_y, int per_z, double *fp) {
    /* neighbour index along each axis for c = -1 (source at +1) and c = +1 */
    int im = i > 0 ? i - 1 : (per_x ? Nx - 1 : 0);
    int ip = i < Nx - 1 ? i + 1 : (per_x ? 0 : Nx - 1);
    int jm = j > 0 ? j - 1 : (per_y ? Ny - 1 : 0);
    int jp = j < Ny - 1 ? j + 1 : (per_y ? 0 : Ny - 1);
    int km = k > 0 ? k - 1 : (per_z ? Nz - 1 : 0);
    int kp = k < Nz - 1 ? k + 1 : (per_z ? 0 : Nz - 1);
    /* "source exists" flags: true when the pull stays inside or wraps */
    int xm = per_x || i > 0, xp = per_x || i < Nx - 1;
    int ym = per_y || j > 0, yp = per_y || j < Ny - 1;
    int zm = per_z || k > 0, zp = per_z || k < Nz - 1;
    fp[0] = f[I3(i, j, k, 0)];
    fp[1] = xm ? f[I3(im, j, k, 1)] : f[I3(i, j, k, 2)];
    fp[2] = xp ? f[I3(ip, j, k, 2)] : f[I3(i, j, k, 1)];
    fp[3] = ym ? f[I3(i, jm, k, 3)] : f[I3(i, j, k, 4)];
    fp[4] = yp ? f[I3(i, jp, k, 4)] : f[I3(i, j, k, 3)];
    fp[5] = zm ? f[I3(i, j, km, 5)] : f[I3(i, j, k, 6)];
    fp[6] = zp ? f[I3(i, j, kp, 6)] : f[I3(i, j, k, 5)];
    fp[7] = (xm && ym) ? f[I3(im, jm, k, 7)] : f[I3(i, j, k, 10)];
    fp[8] = (xp && ym) ? f[I3(ip, jm, k, 8)] : f[I3(i, j, k, 9)];
    fp[9] = (xm && yp) ? f[I3(im, jp, k, 9)] : f[I3(i, j, k, 8)];
    fp[10] = (xp && yp) ? f[I3(ip, jp, k, 10)] : f[I3(i, j, k, 7)];
    fp[11] = (xm && zm) ? f[I3(im, j, km, 11)] : f[I3(i, j, k, 14)];
    fp[12] = (xp && zm) ? f[I3(ip, j, km, 12)] : f[I3(i, j, k, 13)];
    fp[13] = (xm && zp) ? f[I3(im, j, kp, 13)] : f[I3(i, j, k, 12)];
    fp[14] = (xp && zp) ? f[I3(ip, j, kp, 14)] : f[I3(i, j, k, 11)];
    fp[15] = (ym && zm) ? f[I3(i, jm, km, 15)] : f[I3(i, j, k, 18)];
    fp[16] = (yp && zm) ? f[I3(i, jp, km, 16)] : f[I3(i, j, k, 17)];
    fp[17] = (ym && zp) ? f[I3(i, jm, kp, 17)] : f[I3(i, j, k, 16)];
    fp[18] = (yp && zp) ? f[I3(i, jp, kp, 18)] : f[I3(i, j, k, 15)];
}

/* stream_3d!: src/kernels/collide_stream_3d.jl:5-42, 119-123 */
void or_stream_3d(double *f_out, const double *f_in, int Nx, int Ny, int Nz) {
#pragma omp parallel for schedule(static)
    for (int k = 0; k < Nz; ++k)
        for (int j = 0; j < Ny; ++j)
            for (int i = 0; i < Nx; ++i) {
                double fp[19];
                pull3d(f_in, Nx, Ny, Nz, i, j, k, 0, 0, 0, fp);
                for (int q = 0; q < 19; ++q) f_out[I3(i, j, k, q)] = fp[q];
            }
}

static inline void swap_pairs_3d(double *p) {
    static const int a[9] = {1, 3, 5, 7, 8, 11, 12, 15, 16};
    static const int b[9] = {2, 4, 6, 10, 9, 14, 13, 18, 17};
    for (int n = 0; n < 9; ++n) { double t = p[a[n]]; p[a[n]] = p[b[n]]; p[b[n]] = t; }
}

/* collide_3d!: src/kernels/collide_stream_3d.jl:46-103, 137-142 */
void or_collide_3d(double *f, const uint8_t *solid, int Nx, int Ny, int Nz, double omega) {
#pragma omp parallel for schedule(static)
    for (int k = 0; k < Nz; ++k)
        for (int j = 0; j < Ny; ++j)
            for (int i = 0; i < Nx; ++i) {
                double p[19];
                for (int q = 0; q < 19; ++q) p[q] = f[I3(i, j, k, q)];
                if (solid && solid[N3(i, j, k)]) {
                    swap_pairs_3d(p);
                } else {
                    double rho, ux, uy, uz, feq[19];
                    moments3d(p, &rho, &ux, &uy, &uz);
                    double usq = ux * ux + uy * uy + uz * uz;
                    feq3d_all(rho, ux, uy, uz, usq, feq);
                    for (int q = 0; q < 19; ++q) p[q] = p[q] - omega * (p[q] - feq[q]);
                }
                for (int q = 0; q < 19; ++q) f[I3(i, j, k, q)] = p[q];
            }
}

/* compute_macroscopic_3d!: src/kernels/macroscopic.jl:42-80 */
void or_macroscopic_3d(double *rho, double *ux, double *uy, double *uz, const double *f,
                       int Nx, int Ny, int Nz) {
#pragma omp parallel for schedule(static)
    for (int k = 0; k < Nz; ++k)
        for (int j = 0; j < Ny; ++j)
            for (int i = 0; i < Nx; ++i) {
                double p[19];
                for (int q = 0; q < 19; ++q) p[q] = f[I3(i, j, k, q)];
                double r, a, b, c;
                moments3d(p, &r, &a, &b, &c);
                rho[N3(i, j, k)] = r; ux[N3(i, j, k)] = a; uy[N3(i, j, k)] = b; uz[N3(i, j, k)] = c;
            }
}

/* Zou-He velocity face descriptors: src/kernels/boundary_3d.jl:39-137.
 * Face codes: 0 west, 1 east, 2 south, 3 north, 4 bottom, 5 top.
 * Population indices are 0-based here (reference 1-based minus one). */
typedef struct {
    int normal_axis, sign, q_axis, q_axis_opp, q_diag[4], q_diag_opp[4];
    int t1p, t1m, t2p, t2m, parallel[9], outgoing[5];
} or_face3d;

static const or_face3d or_faces[6] = {
    {1, -1, 1, 2, {7, 9, 11, 13}, {10, 8, 14, 12}, 3, 4, 5, 6, {0, 3, 4, 5, 6, 15, 16, 17, 18}, {2, 8, 10, 12, 14}},
    {1, 1, 2, 1, {8, 10, 12, 14}, {9, 7, 13, 11}, 3, 4, 5, 6, {0, 3, 4, 5, 6, 15, 16, 17, 18}, {1, 7, 9, 11, 13}},
    {2, -1, 3, 4, {7, 8, 15, 17}, {10, 9, 18, 16}, 1, 2, 5, 6, {0, 1, 2, 5, 6, 11, 12, 13, 14}, {4, 9, 10, 16, 18}},
    {2, 1, 4, 3, {9, 10, 16, 18}, {8, 7, 17, 15}, 1, 2, 5, 6, {0, 1, 2, 5, 6, 11, 12, 13, 14}, {3, 7, 8, 15, 17}},
    {3, -1, 5, 6, {11, 12, 15, 16}, {14, 13, 18, 17}, 1, 2, 3, 4, {0, 1, 2, 3, 4, 7, 8, 9, 10}, {6, 13, 14, 17, 18}},
    {3, 1, 6, 5, {13, 14, 17, 18}, {12, 11, 16, 15}, 1, 2, 3, 4, {0, 1, 2, 3, 4, 7, 8, 9, 10}, {5, 11, 12, 15, 16}},
};

/* zou_he_velocity_3d_kernel!: src/kernels/boundary_3d.jl:154-223.
 * idx_fixed is 0-based. */
void or_zou_he_velocity_3d(double *f, int Nx, int Ny, int Nz, int face, int idx_fixed,
                           double u_n, double u_t1, double u_t2) {
    const or_face3d *F = &or_faces[face];
    int N1 = F->normal_axis == 1 ? Ny : Nx;
    int N2v = F->normal_axis == 3 ? Ny : Nz;
    for (int b = 0; b < N2v; ++b)
        for (int a = 0; a < N1; ++a) {
            int i, j, k;
            if (F->normal_axis == 1) { i = idx_fixed; j = a; k = b; }
            else if (F->normal_axis == 2) { i = a; j = idx_fixed; k = b; }
            else { i = a; j = b; k = idx_fixed; }
            double sum_par = 0.0, sum_out = 0.0;
            for (int n = 0; n < 9; ++n) sum_par += f[I3(i, j, k, F->parallel[n])];
            for (int n = 0; n < 5; ++n) sum_out += f[I3(i, j, k, F->outgoing[n])];
            double sg = (double)F->sign;
            double denom = 1.0 + sg * u_n;
            double rw = (sum_par + 2.0 * sum_out) / denom;
            f[I3(i, j, k, F->q_axis)] = f[I3(i, j, k, F->q_axis_opp)] - sg * (1.0 / 3.0) * rw * u_n;
            double d1 = f[I3(i, j, k, F->parallel[5])], d2 = f[I3(i, j, k, F->parallel[6])];
            double d3 = f[I3(i, j, k, F->parallel[7])], d4 = f[I3(i, j, k, F->parallel[8])];
            double t1 = (f[I3(i, j, k, F->t1p)] - f[I3(i, j, k, F->t1m)]) + (d1 - d2 + d3 - d4);
            double t2 = (f[I3(i, j, k, F->t2p)] - f[I3(i, j, k, F->t2m)]) + (d1 + d2 - d3 - d4);
            f[I3(i, j, k, F->q_diag[0])] = f[I3(i, j, k, F->q_diag_opp[0])] - 0.5 * t1 + 0.5 * rw * u_t1 - sg * (1.0 / 6.0) * rw * u_n;
            f[I3(i, j, k, F->q_diag[1])] = f[I3(i, j, k, F->q_diag_opp[1])] + 0.5 * t1 - 0.5 * rw * u_t1 - sg * (1.0 / 6.0) * rw * u_n;
            f[I3(i, j, k, F->q_diag[2])] = f[I3(i, j, k, F->q_diag_opp[2])] - 0.5 * t2 + 0.5 * rw * u_t2 - sg * (1.0 / 6.0) * rw * u_n;
            f[I3(i, j, k, F->q_diag[3])] = f[I3(i, j, k, F->q_diag_opp[3])] + 0.5 * t2 - 0.5 * rw * u_t2 - sg * (1.0 / 6.0) * rw * u_n;
        }
}

/* zou_he_pressure_3d_kernel!: src/kernels/boundary_3d.jl:232-288 */
void or_zou_he_pressure_3d(double *f, int Nx, int Ny, int Nz, int face, int idx_fixed,
                           double rho_out) {
    const or_face3d *F = &or_faces[face];
    int N1 = F->normal_axis == 1 ? Ny : Nx;
    int N2v = F->normal_axis == 3 ? Ny : Nz;
    for (int b = 0; b < N2v; ++b)
        for (int a = 0; a < N1; ++a) {
            int i, j, k;
            if (F->normal_axis == 1) { i = idx_fixed; j = a; k = b; }
            else if (F->normal_axis == 2) { i = a; j = idx_fixed; k = b; }
            else { i = a; j = b; k = idx_fixed; }
            double sum_par = 0.0, sum_out = 0.0;
            for (int n = 0; n < 9; ++n) sum_par += f[I3(i, j, k, F->parallel[n])];
            for (int n = 0; n < 5; ++n) sum_out += f[I3(i, j, k, F->outgoing[n])];
            double sg = (double)F->sign;
            double u_n = -sg * (1.0 - (sum_par + 2.0 * sum_out) / rho_out);
            f[I3(i, j, k, F->q_axis)] = f[I3(i, j, k, F->q_axis_opp)] - sg * (1.0 / 3.0) * rho_out * u_n;
            double t1 = f[I3(i, j, k, F->t1p)] - f[I3(i, j, k, F->t1m)];
            double t2 = f[I3(i, j, k, F->t2p)] - f[I3(i, j, k, F->t2m)];
            f[I3(i, j, k, F->q_diag[0])] = f[I3(i, j, k, F->q_diag_opp[0])] - 0.5 * t1 - sg * (1.0 / 6.0) * rho_out * u_n;
            f[I3(i, j, k, F->q_diag[1])] = f[I3(i, j, k, F->q_diag_opp[1])] + 0.5 * t1 - sg * (1.0 / 6.0) * rho_out * u_n;
            f[I3(i, j, k, F->q_diag[2])] = f[I3(i, j, k, F->q_diag_opp[2])] - 0.5 * t2 - sg * (1.0 / 6.0) * rho_out * u_n;
            f[I3(i, j, k, F->q_diag[3])] = f[I3(i, j, k, F->q_diag_opp[3])] + 0.5 * t2 - sg * (1.0 / 6.0) * rho_out * u_n;
        }
}

/* apply_zou_he_top_3d!: src/kernels/boundary_3d.jl:326-330 */
void or_zou_he_top_3d(double *f, double u_wall_x, int Nx, int Ny, int Nz) {
    or_zou_he_velocity_3d(f, Nx, Ny, Nz, 5, Nz - 1, 0.0, u_wall_x, 0.0);
}

/* run_cavity_3d: src/drivers/basic.jl:153-176 */
void or_run_cavity_3d(double *f_a, double *f_b, double *rho, double *ux, double *uy, double *uz,
                      const uint8_t *solid, int Nx, int Ny, int Nz, double omega, double u_lid, int steps) {
    double *fi = f_a, *fo = f_b;
    size_t n = (size_t)Nx * Ny * Nz * 19;
    for (int s = 0; s < steps; ++s) {
        or_stream_3d(fo, fi, Nx, Ny, Nz);
        or_zou_he_top_3d(fo, u_lid, Nx, Ny, Nz);
        or_collide_3d(fo, solid, Nx, Ny, Nz, omega);
        or_macroscopic_3d(rho, ux, uy, uz, fo, Nx, Ny, Nz);
        double *t = fi; fi = fo; fo = t;
    }
    if (fi != f_a) memcpy(f_a, fi, n * sizeof(double));
}

/* Fused D3Q19 TRT step: the DSL spec PullHalfwayBB_3D + SolidInert_3D +
 * Moments_3D + CollideTRTDirect_3D + WriteMoments_3D
 * (src/kernels/li_bb_3d_v2.jl:13-42 with no LI-BB links flagged;
 * bricks_3d.jl:64-230, 476-483).  rho/ux/uy/uz may be NULL: the moment write
 * is then skipped (populations are unaffected). */
void or_fused_trt_3d(double *f_out, const double *f_in, double *rho_o, double *ux_o, double *uy_o,
                     double *uz_o, const uint8_t *solid, int Nx, int Ny, int Nz, double sp, double sm,
                     int per_x, int per_y, int per_z) {
#pragma omp parallel for schedule(static)
    for (int k = 0; k < Nz; ++k)
        for (int j = 0; j < Ny; ++j)
            for (int i = 0; i < Nx; ++i) {
                double p[19];
                size_t n = N3(i, j, k);
                pull3d(f_in, Nx, Ny, Nz, i, j, k, per_x, per_y, per_z, p);
                if (solid && solid[n]) {
                    /* SolidInert_3D: feq_3d(q, 1, 0, 0, 0, 0) = w_q (1 - 1.5*0) */
                    double feq[19];
                    feq3d_all(1.0, 0.0, 0.0, 0.0, 0.0, feq);
                    for (int q = 0; q < 19; ++q) f_out[I3(i, j, k, q)] = feq[q];
                    if (rho_o) { rho_o[n] = 1.0; ux_o[n] = 0.0; uy_o[n] = 0.0; uz_o[n] = 0.0; }
                    continue;
                }
                double rho, ux, uy, uz, feq[19];
                moments3d(p, &rho, &ux, &uy, &uz);
                double usq = ux * ux + uy * uy + uz * uz;
                feq3d_all(rho, ux, uy, uz, usq, feq);
                double a = (sp + sm) * 0.5, b = (sp - sm) * 0.5;
                static const int pa[9] = {1, 3, 5, 7, 8, 11, 12, 15, 16};
                static const int pb[9] = {2, 4, 6, 10, 9, 14, 13, 18, 17};
                f_out[I3(i, j, k, 0)] = p[0] - sp * (p[0] - feq[0]);
                for (int m = 0; m < 9; ++m) {
                    int x = pa[m], y = pb[m];
                    f_out[I3(i, j, k, x)] = p[x] - a * (p[x] - feq[x]) - b * (p[y] - feq[y]);
                    f_out[I3(i, j, k, y)] = p[y] - a * (p[y] - feq[y]) - b * (p[x] - feq[x]);
                }
                if (rho_o) { rho_o[n] = rho; ux_o[n] = ux; uy_o[n] = uy; uz_o[n] = uz; }
            }
}

/* The same fused D3Q19 TRT step in single precision: the reference's
 * T = Float32 path, where every constant is T(literal) and every operation
 * rounds to Float32 (feq_3d: src/kernels/equilibrium_helpers_3d.jl:26-101,
 * moments_3d: :102-112, CollideTRTDirect_3D: src/kernels/dsl/bricks_3d.jl:
 * 179-229).  Same operation order as or_fused_trt_3d.  Used as the timed CPU
 * baseline of the FP32 storages; parity is held by the FP64 restatement. */
static inline float feq_poly_f32(float w, float rho, float cu, float usq) {
    return w * rho * (1.0f + 3.0f * cu + 4.5f * cu * cu - 1.5f * usq);
}

void or_fused_trt_3d_f32(float *f_out, const float *f_in, float *rho_o, float *ux_o,
                         float *uy_o, float *uz_o, const uint8_t *solid, int Nx, int Ny, int Nz,
                         float sp, float sm, int per_x, int per_y, int per_z) {
    const float wr = (float)(1.0 / 3.0), wa = (float)(1.0 / 18.0), we = (float)(1.0 / 36.0);
#pragma omp parallel for schedule(static)
    for (int k = 0; k < Nz; ++k)
        for (int j = 0; j < Ny; ++j)
            for (int i = 0; i < Nx; ++i) {
                float p[19];
                size_t n = N3(i, j, k);
                int im = i > 0 ? i - 1 : (per_x ? Nx - 1 : 0);
                int ip = i < Nx - 1 ? i + 1 : (per_x ? 0 : Nx - 1);
                int jm = j > 0 ? j - 1 : (per_y ? Ny - 1 : 0);
                int jp = j < Ny - 1 ? j + 1 : (per_y ? 0 : Ny - 1);
                int km = k > 0 ? k - 1 : (per_z ? Nz - 1 : 0);
                int kp = k < Nz - 1 ? k + 1 : (per_z ? 0 : Nz - 1);
                int xm = per_x || i > 0, xp = per_x || i < Nx - 1;
                int ym = per_y || j > 0, yp = per_y || j < Ny - 1;
                int zm = per_z || k > 0, zp = per_z || k < Nz - 1;
                p[0] = f_in[I3(i, j, k, 0)];
                p[1] = xm ? f_in[I3(im, j, k, 1)] : f_in[I3(i, j, k, 2)];
                p[2] = xp ? f_in[I3(ip, j, k, 2)] : f_in[I3(i, j, k, 1)];
                p[3] = ym ? f_in[I3(i, jm, k, 3)] : f_in[I3(i, j, k, 4)];
                p[4] = yp ? f_in[I3(i, jp, k, 4)] : f_in[I3(i, j, k, 3)];
                p[5] = zm ? f_in[I3(i, j, km, 5)] : f_in[I3(i, j, k, 6)];
                p[6] = zp ? f_in[I3(i, j, kp, 6)] : f_in[I3(i, j, k, 5)];
                p[7] = (xm && ym) ? f_in[I3(im, jm, k, 7)] : f_in[I3(i, j, k, 10)];
                p[8] = (xp && ym) ? f_in[I3(ip, jm, k, 8)] : f_in[I3(i, j, k, 9)];
                p[9] = (xm && yp) ? f_in[I3(im, jp, k, 9)] : f_in[I3(i, j, k, 8)];
                p[10] = (xp && yp) ? f_in[I3(ip, jp, k, 10)] : f_in[I3(i, j, k, 7)];
                p[11] = (xm && zm) ? f_in[I3(im, j, km, 11)] : f_in[I3(i, j, k, 14)];
                p[12] = (xp && zm) ? f_in[I3(ip, j, km, 12)] : f_in[I3(i, j, k, 13)];
                p[13] = (xm && zp) ? f_in[I3(im, j, kp, 13)] : f_in[I3(i, j, k, 12)];
                p[14] = (xp && zp) ? f_in[I3(ip, j, kp, 14)] : f_in[I3(i, j, k, 11)];
                p[15] = (ym && zm) ? f_in[I3(i, jm, km, 15)] : f_in[I3(i, j, k, 18)];
                p[16] = (yp && zm) ? f_in[I3(i, jp, km, 16)] : f_in[I3(i, j, k, 17)];
                p[17] = (ym && zp) ? f_in[I3(i, jm, kp, 17)] : f_in[I3(i, j, k, 16)];
                p[18] = (yp && zp) ? f_in[I3(i, jp, kp, 18)] : f_in[I3(i, j, k, 15)];
                if (solid && solid[n]) {
                    for (int q = 0; q < 19; ++q)
                        f_out[I3(i, j, k, q)] = q == 0 ? wr * 1.0f * (1.0f - 1.5f * 0.0f)
                                                       : feq_poly_f32(q < 7 ? wa : we, 1.0f, 0.0f, 0.0f);
                    if (rho_o) { rho_o[n] = 1.0f; ux_o[n] = 0.0f; uy_o[n] = 0.0f; uz_o[n] = 0.0f; }
                    continue;
                }
                float r = p[0] + p[1] + p[2] + p[3] + p[4] + p[5] + p[6] + p[7] + p[8] + p[9] +
                          p[10] + p[11] + p[12] + p[13] + p[14] + p[15] + p[16] + p[17] + p[18];
                float inv = 1.0f / r;
                float ux = (p[1] - p[2] + p[7] - p[8] + p[9] - p[10] + p[11] - p[12] + p[13] - p[14]) * inv;
                float uy = (p[3] - p[4] + p[7] + p[8] - p[9] - p[10] + p[15] - p[16] + p[17] - p[18]) * inv;
                float uz = (p[5] - p[6] + p[11] + p[12] - p[13] - p[14] + p[15] + p[16] - p[17] - p[18]) * inv;
                float usq = ux * ux + uy * uy + uz * uz;
                float feq[19];
                feq[0] = wr * r * (1.0f - 1.5f * usq);
                feq[1] = feq_poly_f32(wa, r, ux, usq);
                feq[2] = feq_poly_f32(wa, r, -ux, usq);
                feq[3] = feq_poly_f32(wa, r, uy, usq);
                feq[4] = feq_poly_f32(wa, r, -uy, usq);
                feq[5] = feq_poly_f32(wa, r, uz, usq);
                feq[6] = feq_poly_f32(wa, r, -uz, usq);
                feq[7] = feq_poly_f32(we, r, ux + uy, usq);
                feq[8] = feq_poly_f32(we, r, -ux + uy, usq);
                feq[9] = feq_poly_f32(we, r, ux - uy, usq);
                feq[10] = feq_poly_f32(we, r, -ux - uy, usq);
                feq[11] = feq_poly_f32(we, r, ux + uz, usq);
                feq[12] = feq_poly_f32(we, r, -ux + uz, usq);
                feq[13] = feq_poly_f32(we, r, ux - uz, usq);
                feq[14] = feq_poly_f32(we, r, -ux - uz, usq);
                feq[15] = feq_poly_f32(we, r, uy + uz, usq);
                feq[16] = feq_poly_f32(we, r, -uy + uz, usq);
                feq[17] = feq_poly_f32(we, r, uy - uz, usq);
                feq[18] = feq_poly_f32(we, r, -uy - uz, usq);
                float a = (sp + sm) * 0.5f, b = (sp - sm) * 0.5f;
                static const int pa[9] = {1, 3, 5, 7, 8, 11, 12, 15, 16};
                static const int pb[9] = {2, 4, 6, 10, 9, 14, 13, 18, 17};
                f_out[I3(i, j, k, 0)] = p[0] - sp * (p[0] - feq[0]);
                for (int m = 0; m < 9; ++m) {
                    int x = pa[m], y = pb[m];
                    f_out[I3(i, j, k, x)] = p[x] - a * (p[x] - feq[x]) - b * (p[y] - feq[y]);
                    f_out[I3(i, j, k, y)] = p[y] - a * (p[y] - feq[y]) - b * (p[x] - feq[x]);
                }
                if (rho_o) { rho_o[n] = r; ux_o[n] = ux; uy_o[n] = uy; uz_o[n] = uz; }
            }
}

/* stream_periodic_xz_movingwall_y_3d!: src/kernels/stream_periodic_3d.jl:106-186 */
void or_stream_periodic_xz_movingwall_y_3d(double *f_out, const double *f_in, double Ub, double Ut,
                                           double rho_w, int Nx, int Ny, int Nz) {
#pragma omp parallel for schedule(static)
    for (int k = 0; k < Nz; ++k)
        for (int j = 0; j < Ny; ++j)
            for (int i = 0; i < Nx; ++i) {
                int im = i > 0 ? i - 1 : Nx - 1, ip = i < Nx - 1 ? i + 1 : 0;
                int km = k > 0 ? k - 1 : Nz - 1, kp = k < Nz - 1 ? k + 1 : 0;
                int lo = j == 0, hi = j == Ny - 1;
                int jm1 = j > 0 ? j - 1 : j, jp1 = j < Ny - 1 ? j + 1 : j;
                double cbot = 1.0 / 6.0 * rho_w * Ub, ctop = 1.0 / 6.0 * rho_w * Ut;
                f_out[I3(i, j, k, 0)] = f_in[I3(i, j, k, 0)];
                f_out[I3(i, j, k, 1)] = f_in[I3(im, j, k, 1)];
                f_out[I3(i, j, k, 2)] = f_in[I3(ip, j, k, 2)];
                f_out[I3(i, j, k, 3)] = lo ? f_in[I3(i, j, k, 4)] : f_in[I3(i, jm1, k, 3)];
                f_out[I3(i, j, k, 4)] = hi ? f_in[I3(i, j, k, 3)] : f_in[I3(i, jp1, k, 4)];
                f_out[I3(i, j, k, 5)] = f_in[I3(i, j, km, 5)];
                f_out[I3(i, j, k, 6)] = f_in[I3(i, j, kp, 6)];
                f_out[I3(i, j, k, 7)] = lo ? f_in[I3(i, j, k, 10)] + cbot : f_in[I3(im, jm1, k, 7)];
                f_out[I3(i, j, k, 8)] = lo ? f_in[I3(i, j, k, 9)] - cbot : f_in[I3(ip, jm1, k, 8)];
                f_out[I3(i, j, k, 9)] = hi ? f_in[I3(i, j, k, 8)] + ctop : f_in[I3(im, jp1, k, 9)];
                f_out[I3(i, j, k, 10)] = hi ? f_in[I3(i, j, k, 7)] - ctop : f_in[I3(ip, jp1, k, 10)];
                f_out[I3(i, j, k, 11)] = f_in[I3(im, j, km, 11)];
                f_out[I3(i, j, k, 12)] = f_in[I3(ip, j, km, 12)];
                f_out[I3(i, j, k, 13)] = f_in[I3(im, j, kp, 13)];
                f_out[I3(i, j, k, 14)] = f_in[I3(ip, j, kp, 14)];
                f_out[I3(i, j, k, 15)] = lo ? f_in[I3(i, j, k, 18)] : f_in[I3(i, jm1, km, 15)];
                f_out[I3(i, j, k, 16)] = hi ? f_in[I3(i, j, k, 17)] : f_in[I3(i, jp1, km, 16)];
                f_out[I3(i, j, k, 17)] = lo ? f_in[I3(i, j, k, 16)] : f_in[I3(i, jm1, kp, 17)];
                f_out[I3(i, j, k, 18)] = hi ? f_in[I3(i, j, k, 15)] : f_in[I3(i, jp1, kp, 18)];
            }
}

/* ------------------------------------------------------------------------ */
/* Thermal double distribution: src/kernels/fused_thermal_2d.jl             */
/* ------------------------------------------------------------------------ */

/* apply_thermal_bc_cavity: fused_thermal_2d.jl:37-57 */
static inline void thermal_bc(double *g, int i, int Nx, double T_hot, double T_cold) {
    if (i == 0) {
        g[1] = -g[1] + 2.0 * (1.0 / 9.0) * T_hot;
        g[5] = -g[5] + 2.0 * (1.0 / 36.0) * T_hot;
        g[8] = -g[8] + 2.0 * (1.0 / 36.0) * T_hot;
    }
    if (i == Nx - 1) {
        g[3] = -g[3] + 2.0 * (1.0 / 9.0) * T_cold;
        g[6] = -g[6] + 2.0 * (1.0 / 36.0) * T_cold;
        g[7] = -g[7] + 2.0 * (1.0 / 36.0) * T_cold;
    }
}

/* collide_thermal_node: fused_thermal_2d.jl:76-111 */
static inline void collide_thermal(double *g, double ux, double uy, double wT) {
    double Tm = g[0] + g[1] + g[2] + g[3] + g[4] + g[5] + g[6] + g[7] + g[8];
    const double t3 = 3.0;
    double geq;
    geq = 4.0 / 9.0 * Tm;                              g[0] = g[0] - wT * (g[0] - geq);
    geq = 1.0 / 9.0 * Tm * (1.0 + t3 * ux);            g[1] = g[1] - wT * (g[1] - geq);
    geq = 1.0 / 9.0 * Tm * (1.0 + t3 * uy);            g[2] = g[2] - wT * (g[2] - geq);
    geq = 1.0 / 9.0 * Tm * (1.0 - t3 * ux);            g[3] = g[3] - wT * (g[3] - geq);
    geq = 1.0 / 9.0 * Tm * (1.0 - t3 * uy);            g[4] = g[4] - wT * (g[4] - geq);
    geq = 1.0 / 36.0 * Tm * (1.0 + t3 * (ux + uy));    g[5] = g[5] - wT * (g[5] - geq);
    geq = 1.0 / 36.0 * Tm * (1.0 + t3 * (-ux + uy));   g[6] = g[6] - wT * (g[6] - geq);
    geq = 1.0 / 36.0 * Tm * (1.0 + t3 * (-ux - uy));   g[7] = g[7] - wT * (g[7] - geq);
    geq = 1.0 / 36.0 * Tm * (1.0 + t3 * (ux - uy));    g[8] = g[8] - wT * (g[8] - geq);
}

/* collide_boussinesq_node: fused_thermal_2d.jl:115-151 */
static inline void collide_boussinesq(double *f, double rho, double ux, double uy, double fy, double w) {
    const double fx = 0.0;
    double usq = ux * ux + uy * uy;
    double gp = 1.0 - w / 2.0;
    const double t3 = 3.0;
    double feq[9], S[9];
    feq2d_all(rho, ux, uy, usq, feq);
    S[0] = 4.0 / 9.0 * ((-ux) * fx + (-uy) * fy) * t3;
    S[1] = 1.0 / 9.0 * ((1.0 - ux) * fx + (-uy) * fy) * t3 + 1.0 / 9.0 * ux * fx * 9.0;
    S[2] = 1.0 / 9.0 * ((-ux) * fx + (1.0 - uy) * fy) * t3 + 1.0 / 9.0 * uy * fy * 9.0;
    S[3] = 1.0 / 9.0 * ((-1.0 - ux) * fx + (-uy) * fy) * t3 + 1.0 / 9.0 * ux * fx * 9.0;
    S[4] = 1.0 / 9.0 * ((-ux) * fx + (-1.0 - uy) * fy) * t3 + 1.0 / 9.0 * uy * fy * 9.0;
    S[5] = 1.0 / 36.0 * ((1.0 - ux) * fx + (1.0 - uy) * fy) * t3 + 1.0 / 36.0 * (ux + uy) * (fx + fy) * 9.0;
    S[6] = 1.0 / 36.0 * ((-1.0 - ux) * fx + (1.0 - uy) * fy) * t3 + 1.0 / 36.0 * (-ux + uy) * (-fx + fy) * 9.0;
    S[7] = 1.0 / 36.0 * ((-1.0 - ux) * fx + (-1.0 - uy) * fy) * t3 + 1.0 / 36.0 * (-ux - uy) * (-fx - fy) * 9.0;
    S[8] = 1.0 / 36.0 * ((1.0 - ux) * fx + (-1.0 - uy) * fy) * t3 + 1.0 / 36.0 * (ux - uy) * (fx - fy) * 9.0;
    for (int q = 0; q < 9; ++q) f[q] = f[q] - w * (f[q] - feq[q]) + gp * S[q];
}

/* fused_natconv_step! (and _vt_ when visc_var != 0):
 * src/kernels/fused_thermal_2d.jl:178-238, 251-278. */
static void natconv_core(double *f_out, const double *f_in, double *g_out, const double *g_in,
                         double *Temp, int Nx, int Ny, double w_f, double w_T, double beta_g,
                         double T_ref, double T_hot, double T_cold, int visc_var, double nu_ref,
                         double T0_visc, double a_visc) {
#pragma omp parallel for schedule(static)
    for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i) {
            double fp[9], gp[9];
            pull2d(f_in, Nx, Ny, i, j, fp);
            pull2d(g_in, Nx, Ny, i, j, gp);
            thermal_bc(gp, i, Nx, T_hot, T_cold);
            double Tl = gp[0] + gp[1] + gp[2] + gp[3] + gp[4] + gp[5] + gp[6] + gp[7] + gp[8];
            Temp[N2(i, j)] = Tl;
            double fy = beta_g * (Tl - T_ref);
            double rho = fp[0] + fp[1] + fp[2] + fp[3] + fp[4] + fp[5] + fp[6] + fp[7] + fp[8];
            double inv = 1.0 / rho;
            double ux = (fp[1] - fp[3] + fp[5] - fp[6] - fp[7] + fp[8]) * inv;
            double uy = ((fp[2] - fp[4] + fp[5] + fp[6] - fp[7] - fp[8]) + fy / 2.0) * inv;
            collide_thermal(gp, ux, uy, w_T);
            for (int q = 0; q < 9; ++q) g_out[I2(i, j, q)] = gp[q];
            double w = w_f;
            if (visc_var) {
                double nul = nu_ref * exp(a_visc * (Tl - T0_visc));
                w = 1.0 / (3.0 * nul + 0.5);
            }
            collide_boussinesq(fp, rho, ux, uy, fy, w);
            for (int q = 0; q < 9; ++q) f_out[I2(i, j, q)] = fp[q];
        }
}

void or_fused_natconv_2d(double *f_out, const double *f_in, double *g_out, const double *g_in,
                         double *Temp, int Nx, int Ny, double w_f, double w_T, double beta_g,
                         double T_ref, double T_hot, double T_cold) {
    natconv_core(f_out, f_in, g_out, g_in, Temp, Nx, Ny, w_f, w_T, beta_g, T_ref, T_hot, T_cold,
                 0, 0.0, 0.0, 0.0);
}

void or_fused_natconv_vt_2d(double *f_out, const double *f_in, double *g_out, const double *g_in,
                            double *Temp, int Nx, int Ny, double nu_ref, double T0_visc,
                            double a_visc, double w_T, double beta_g, double T_ref, double T_hot,
                            double T_cold) {
    natconv_core(f_out, f_in, g_out, g_in, Temp, Nx, Ny, 0.0, w_T, beta_g, T_ref, T_hot, T_cold,
                 1, nu_ref, T0_visc, a_visc);
}

/* compute_temperature_2d!: src/kernels/thermal_2d.jl:113-138 (T = sum g). */
void or_temperature_2d(double *Temp, const double *g, int Nx, int Ny) {
    for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i) {
            double s = g[I2(i, j, 0)] + g[I2(i, j, 1)] + g[I2(i, j, 2)] + g[I2(i, j, 3)] +
                       g[I2(i, j, 4)] + g[I2(i, j, 5)] + g[I2(i, j, 6)] + g[I2(i, j, 7)] + g[I2(i, j, 8)];
            Temp[N2(i, j)] = s;
        }
}

/* Steady residual over fluid nodes, r_u = ||u - u_prev||_2 / ||u||_2
 * (src/drivers/gnf_periodic_steady.jl:186-194), sequential FP64 sums.
 * ndim = 2 or 3; uz/uz_prev ignored for 2. */
double or_residual(const double *ux, const double *uy, const double *uz, const double *uxp,
                   const double *uyp, const double *uzp, const uint8_t *solid, size_t n, int ndim) {
    double du2 = 0.0, u2 = 0.0;
    for (size_t m = 0; m < n; ++m) {
        if (solid && solid[m]) continue;
        double a = ux[m] - uxp[m], b = uy[m] - uyp[m];
        double d = a * a + b * b, s = ux[m] * ux[m] + uy[m] * uy[m];
        if (ndim == 3) { double c = uz[m] - uzp[m]; d += c * c; s += uz[m] * uz[m]; }
        du2 += d; u2 += s;
    }
    return sqrt(du2 / u2);
}

int or_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void or_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ------------------------------------------------------------------------ */
/* Unfused thermal DDF: src/kernels/thermal_2d.jl, src/kernels/thermal_3d.jl */
/* ------------------------------------------------------------------------ */

/* collide_thermal_2d!: thermal_2d.jl:16-81 */
void or_collide_thermal_2d(double *g, const double *ux, const double *uy, int Nx, int Ny,
                           double wT) {
    for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i) {
            double p[9];
            for (int q = 0; q < 9; ++q) p[q] = g[I2(i, j, q)];
            collide_thermal(p, ux[N2(i, j)], uy[N2(i, j)], wT);
            for (int q = 0; q < 9; ++q) g[I2(i, j, q)] = p[q];
        }
}

/* collide_thermal_masked_2d!: thermal_2d.jl:83-109 (per-population loop
 * with w_q and c_q selected per q, skipped nodes untouched) */
void or_collide_thermal_masked_2d(double *g, const double *ux, const double *uy,
                                  const uint8_t *skip, int Nx, int Ny, double wT) {
    for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i) {
            if (skip && skip[N2(i, j)]) continue;
            double a = ux[N2(i, j)], b = uy[N2(i, j)];
            double Tm = g[I2(i, j, 0)] + g[I2(i, j, 1)] + g[I2(i, j, 2)] + g[I2(i, j, 3)] +
                        g[I2(i, j, 4)] + g[I2(i, j, 5)] + g[I2(i, j, 6)] + g[I2(i, j, 7)] +
                        g[I2(i, j, 8)];
            for (int q = 0; q < 9; ++q) {
                double w = q == 0 ? 4.0 / 9.0 : (q <= 4 ? 1.0 / 9.0 : 1.0 / 36.0);
                double geq = w * Tm * (1.0 + 3.0 * ((double)or_d2q9_cx[q] * a +
                                                    (double)or_d2q9_cy[q] * b));
                g[I2(i, j, q)] -= wT * (g[I2(i, j, q)] - geq);
            }
        }
}

/* _abb_slot: thermal_2d.jl:163-166 */
static inline double abb_slot(double gq, double w2, double T_face, int on_corner, double T_corner,
                              int skip) {
    double T_link = on_corner ? T_corner : T_face;
    return (on_corner && skip) ? gq : -gq + w2 * T_link;
}

/* _fixed_temp_{west,east,south,north}_2d!: thermal_2d.jl:174-292
 * face 0 west, 1 east, 2 south, 3 north; Tc/skip at the low / high end. */
void or_fixed_temp_face_2d(double *g, int Nx, int Ny, int face, double T_wall, double Tc_lo,
                           double Tc_hi, int skip_lo, int skip_hi) {
    const double wa = 2.0 * (1.0 / 9.0), we = 2.0 * (1.0 / 36.0);
    if (face == 2) {          /* south, j = 0: slots 3, 6, 7 (reference) */
        for (int i = 0; i < Nx; ++i) {
            g[I2(i, 0, 2)] = -g[I2(i, 0, 2)] + wa * T_wall;
            g[I2(i, 0, 5)] = abb_slot(g[I2(i, 0, 5)], we, T_wall, i == 0, Tc_lo, skip_lo);
            g[I2(i, 0, 6)] = abb_slot(g[I2(i, 0, 6)], we, T_wall, i == Nx - 1, Tc_hi, skip_hi);
        }
    } else if (face == 3) {   /* north, j = Ny-1: slots 5, 9, 8 */
        int j = Ny - 1;
        for (int i = 0; i < Nx; ++i) {
            g[I2(i, j, 4)] = -g[I2(i, j, 4)] + wa * T_wall;
            g[I2(i, j, 8)] = abb_slot(g[I2(i, j, 8)], we, T_wall, i == 0, Tc_lo, skip_lo);
            g[I2(i, j, 7)] = abb_slot(g[I2(i, j, 7)], we, T_wall, i == Nx - 1, Tc_hi, skip_hi);
        }
    } else if (face == 0) {   /* west, i = 0: slots 2, 6, 9 */
        for (int j = 0; j < Ny; ++j) {
            g[I2(0, j, 1)] = -g[I2(0, j, 1)] + wa * T_wall;
            g[I2(0, j, 5)] = abb_slot(g[I2(0, j, 5)], we, T_wall, j == 0, Tc_lo, skip_lo);
            g[I2(0, j, 8)] = abb_slot(g[I2(0, j, 8)], we, T_wall, j == Ny - 1, Tc_hi, skip_hi);
        }
    } else {                  /* east, i = Nx-1: slots 4, 7, 8 */
        int i = Nx - 1;
        for (int j = 0; j < Ny; ++j) {
            g[I2(i, j, 3)] = -g[I2(i, j, 3)] + wa * T_wall;
            g[I2(i, j, 6)] = abb_slot(g[I2(i, j, 6)], we, T_wall, j == 0, Tc_lo, skip_lo);
            g[I2(i, j, 7)] = abb_slot(g[I2(i, j, 7)], we, T_wall, j == Ny - 1, Tc_hi, skip_hi);
        }
    }
}

/* _corner_temp: thermal_2d.jl:356-357 */
static inline double corner_temp(double Ta, int has_b, double Tb) {
    return has_b ? (Ta + Tb) / 2.0 : Ta;
}

/* _apply_fixed_temp_faces_2d!: thermal_2d.jl:371-392, faces in the order
 * west, east, south, north; bit n of `faces` = face n Dirichlet at T[n]. */
void or_fixed_temp_2d(double *g, int Nx, int Ny, unsigned faces, const double *T) {
    int hw = faces & 1u, he = (faces >> 1) & 1u, hs = (faces >> 2) & 1u, hn = (faces >> 3) & 1u;
    if (hw) or_fixed_temp_face_2d(g, Nx, Ny, 0, T[0], corner_temp(T[0], hs, T[2]),
                                  corner_temp(T[0], hn, T[3]), 0, 0);
    if (he) or_fixed_temp_face_2d(g, Nx, Ny, 1, T[1], corner_temp(T[1], hs, T[2]),
                                  corner_temp(T[1], hn, T[3]), 0, 0);
    if (hs) or_fixed_temp_face_2d(g, Nx, Ny, 2, T[2], T[2], T[2], hw, he);
    if (hn) or_fixed_temp_face_2d(g, Nx, Ny, 3, T[3], T[3], T[3], hw, he);
}

/* collide_boussinesq_2d! (thermal_2d.jl:421-473) and the nu(T) kernels:
 * mode 1 collide_boussinesq_vt_2d! (:482-539, Arrhenius), mode 2
 * collide_boussinesq_vt_modified_2d! (:593-650). */
void or_collide_boussinesq_2d(double *f, const double *Temp, const uint8_t *solid, int Nx, int Ny,
                              int mode, double omega, double nu_ref, double Ta, double Aa,
                              double beta_g, double T_ref) {
    for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i) {
            double p[9];
            for (int q = 0; q < 9; ++q) p[q] = f[I2(i, j, q)];
            if (solid && solid[N2(i, j)]) {
                swap_pairs_2d(p);
            } else {
                double Tl = Temp[N2(i, j)];
                double w = omega;
                if (mode == 1) {
                    double nul = nu_ref * exp(Aa * (1.0 / Tl - 1.0 / Ta));
                    w = 1.0 / (3.0 * nul + 0.5);
                } else if (mode == 2) {
                    double nul = nu_ref * exp(Aa * (Tl - Ta));
                    w = 1.0 / (3.0 * nul + 0.5);
                }
                double fy = beta_g * (Tl - T_ref);
                double fx = 0.0;
                double rho = p[0] + p[1] + p[2] + p[3] + p[4] + p[5] + p[6] + p[7] + p[8];
                double inv = 1.0 / rho;
                double ux = ((p[1] - p[3] + p[5] - p[6] - p[7] + p[8]) + fx / 2.0) * inv;
                double uy = ((p[2] - p[4] + p[5] + p[6] - p[7] - p[8]) + fy / 2.0) * inv;
                collide_boussinesq(p, rho, ux, uy, fy, w);
            }
            for (int q = 0; q < 9; ++q) f[I2(i, j, q)] = p[q];
        }
}

/* collide_thermal_3d!: thermal_3d.jl:12-124 */
void or_collide_thermal_3d(double *g, const double *ux, const double *uy, const double *uz,
                           int Nx, int Ny, int Nz, double wT) {
    for (int k = 0; k < Nz; ++k)
        for (int j = 0; j < Ny; ++j)
            for (int i = 0; i < Nx; ++i) {
                double p[19];
                for (int q = 0; q < 19; ++q) p[q] = g[I3(i, j, k, q)];
                double Tm = p[0] + p[1] + p[2] + p[3] + p[4] + p[5] + p[6] + p[7] + p[8] + p[9] +
                            p[10] + p[11] + p[12] + p[13] + p[14] + p[15] + p[16] + p[17] + p[18];
                double a = ux[N3(i, j, k)], b = uy[N3(i, j, k)], c = uz[N3(i, j, k)];
                const double t3 = 3.0, wa = 1.0 / 18.0, we = 1.0 / 36.0;
                double geq[19];
                geq[0] = 1.0 / 3.0 * Tm;
                geq[1] = wa * Tm * (1.0 + t3 * a);
                geq[2] = wa * Tm * (1.0 - t3 * a);
                geq[3] = wa * Tm * (1.0 + t3 * b);
                geq[4] = wa * Tm * (1.0 - t3 * b);
                geq[5] = wa * Tm * (1.0 + t3 * c);
                geq[6] = wa * Tm * (1.0 - t3 * c);
                geq[7] = we * Tm * (1.0 + t3 * (a + b));
                geq[8] = we * Tm * (1.0 + t3 * (-a + b));
                geq[9] = we * Tm * (1.0 + t3 * (a - b));
                geq[10] = we * Tm * (1.0 + t3 * (-a - b));
                geq[11] = we * Tm * (1.0 + t3 * (a + c));
                geq[12] = we * Tm * (1.0 + t3 * (-a + c));
                geq[13] = we * Tm * (1.0 + t3 * (a - c));
                geq[14] = we * Tm * (1.0 + t3 * (-a - c));
                geq[15] = we * Tm * (1.0 + t3 * (b + c));
                geq[16] = we * Tm * (1.0 + t3 * (-b + c));
                geq[17] = we * Tm * (1.0 + t3 * (b - c));
                geq[18] = we * Tm * (1.0 + t3 * (-b - c));
                for (int q = 0; q < 19; ++q) g[I3(i, j, k, q)] = p[q] - wT * (p[q] - geq[q]);
            }
}

/* compute_temperature_3d!: thermal_3d.jl:128-155 */
void or_temperature_3d(double *Temp, const double *g, int Nx, int Ny, int Nz) {
    for (int k = 0; k < Nz; ++k)
        for (int j = 0; j < Ny; ++j)
            for (int i = 0; i < Nx; ++i) {
                double s = g[I3(i, j, k, 0)];
                for (int q = 1; q < 19; ++q) s = s + g[I3(i, j, k, q)];
                Temp[N3(i, j, k)] = s;
            }
}

/* _fixed_temp_<face>_3d!: thermal_3d.jl:193-480.  For each face, the main
 * slot and the four edge slots with the test that puts a node on that edge,
 * as listed in the reference kernels (0-based slots). */
void or_fixed_temp_face_3d(double *g, int Nx, int Ny, int Nz, int face, double T_wall,
                           const double *T_e, unsigned skip) {
    static const int main_q[6] = {1, 2, 3, 4, 5, 6};
    static const int edge_q[6][4] = {{7, 9, 11, 13}, {8, 10, 12, 14}, {7, 8, 15, 17},
                                     {9, 10, 16, 18}, {11, 12, 15, 16}, {13, 14, 17, 18}};
    const double wa = 2.0 * (1.0 / 18.0), we = 2.0 * (1.0 / 36.0);
    for (int k = 0; k < Nz; ++k)
        for (int j = 0; j < Ny; ++j)
            for (int i = 0; i < Nx; ++i) {
                int on_face, e[4];
                switch (face) {
                case 0: on_face = i == 0; e[0] = j == 0; e[1] = j == Ny - 1; e[2] = k == 0; e[3] = k == Nz - 1; break;
                case 1: on_face = i == Nx - 1; e[0] = j == 0; e[1] = j == Ny - 1; e[2] = k == 0; e[3] = k == Nz - 1; break;
                case 2: on_face = j == 0; e[0] = i == 0; e[1] = i == Nx - 1; e[2] = k == 0; e[3] = k == Nz - 1; break;
                case 3: on_face = j == Ny - 1; e[0] = i == 0; e[1] = i == Nx - 1; e[2] = k == 0; e[3] = k == Nz - 1; break;
                case 4: on_face = k == 0; e[0] = i == 0; e[1] = i == Nx - 1; e[2] = j == 0; e[3] = j == Ny - 1; break;
                default: on_face = k == Nz - 1; e[0] = i == 0; e[1] = i == Nx - 1; e[2] = j == 0; e[3] = j == Ny - 1; break;
                }
                if (!on_face) continue;
                size_t m = I3(i, j, k, main_q[face]);
                g[m] = -g[m] + wa * T_wall;
                for (int n = 0; n < 4; ++n) {
                    size_t s = I3(i, j, k, edge_q[face][n]);
                    g[s] = abb_slot(g[s], we, T_wall, e[n], T_e[n], (skip >> n) & 1u);
                }
            }
}

/* _apply_fixed_temp_faces_3d!: thermal_3d.jl:494-533, faces in the order
 * west, east, south, north, bottom, top. */
void or_fixed_temp_3d(double *g, int Nx, int Ny, int Nz, unsigned faces, const double *T) {
    int h[6];
    for (int n = 0; n < 6; ++n) h[n] = (faces >> n) & 1u;
    for (int face = 0; face < 6; ++face) {
        if (!h[face]) continue;
        double Te[4];
        unsigned skip = 0;
        double t = T[face];
        if (face < 2) {
            Te[0] = corner_temp(t, h[2], T[2]); Te[1] = corner_temp(t, h[3], T[3]);
            Te[2] = corner_temp(t, h[4], T[4]); Te[3] = corner_temp(t, h[5], T[5]);
        } else if (face < 4) {
            Te[0] = t; Te[1] = t;
            Te[2] = corner_temp(t, h[4], T[4]); Te[3] = corner_temp(t, h[5], T[5]);
            skip = (unsigned)h[0] | ((unsigned)h[1] << 1);
        } else {
            Te[0] = Te[1] = Te[2] = Te[3] = t;
            skip = (unsigned)h[0] | ((unsigned)h[1] << 1) | ((unsigned)h[2] << 2) | ((unsigned)h[3] << 3);
        }
        or_fixed_temp_face_3d(g, Nx, Ny, Nz, face, t, Te, skip);
    }
}

/* collide_boussinesq_3d!: thermal_3d.jl:559-733, population by population
 * as the reference writes them (F = (0, beta_g (T - T_ref), 0)). */
/* Shared by collide_boussinesq_3d! (mode 0: F = (0, beta_g (T - T_ref), 0)) and
 * collide_guo_3d! / collide_guo_field_3d! (src/kernels/collide_guo_3d.jl:5-186,
 * 199-323; mode 1 constant F, mode 2 per-node fields): the same expressions. */
static void guo_3d_core(double *f, const double *Temp, const uint8_t *solid, int Nx, int Ny,
                        int Nz, double omega, double beta_g, double T_ref, int mode, double Fx,
                        double Fy, double Fz, const double *Fxf, const double *Fyf,
                        const double *Fzf);

void or_collide_boussinesq_3d(double *f, const double *Temp, const uint8_t *solid, int Nx, int Ny,
                              int Nz, double omega, double beta_g, double T_ref) {
    guo_3d_core(f, Temp, solid, Nx, Ny, Nz, omega, beta_g, T_ref, 0, 0.0, 0.0, 0.0, NULL, NULL,
                NULL);
}

void or_collide_guo_3d(double *f, const uint8_t *solid, int Nx, int Ny, int Nz, double omega,
                       double Fx, double Fy, double Fz) {
    guo_3d_core(f, NULL, solid, Nx, Ny, Nz, omega, 0.0, 0.0, 1, Fx, Fy, Fz, NULL, NULL, NULL);
}

void or_collide_guo_field_3d(double *f, const uint8_t *solid, const double *Fxf,
                             const double *Fyf, const double *Fzf, int Nx, int Ny, int Nz,
                             double omega) {
    guo_3d_core(f, NULL, solid, Nx, Ny, Nz, omega, 0.0, 0.0, 2, 0.0, 0.0, 0.0, Fxf, Fyf, Fzf);
}

static void guo_3d_core(double *f, const double *Temp, const uint8_t *solid, int Nx, int Ny,
                        int Nz, double omega, double beta_g, double T_ref, int mode, double Fx,
                        double Fy, double Fz, const double *Fxf, const double *Fyf,
                        const double *Fzf) {
    for (int k = 0; k < Nz; ++k)
        for (int j = 0; j < Ny; ++j)
            for (int i = 0; i < Nx; ++i) {
                double p[19];
                for (int q = 0; q < 19; ++q) p[q] = f[I3(i, j, k, q)];
                if (solid && solid[N3(i, j, k)]) {
                    swap_pairs_3d(p);
                } else {
                    size_t nn = N3(i, j, k);
                    double fx = mode == 0 ? 0.0 : (mode == 1 ? Fx : Fxf[nn]);
                    double fy = mode == 0 ? beta_g * (Temp[nn] - T_ref) : (mode == 1 ? Fy : Fyf[nn]);
                    double fz = mode == 0 ? 0.0 : (mode == 1 ? Fz : Fzf[nn]);
                    double rho = p[0] + p[1] + p[2] + p[3] + p[4] + p[5] + p[6] + p[7] + p[8] +
                                 p[9] + p[10] + p[11] + p[12] + p[13] + p[14] + p[15] + p[16] +
                                 p[17] + p[18];
                    double inv = 1.0 / rho;
                    double ux = ((p[1] - p[2] + p[7] - p[8] + p[9] - p[10] + p[11] - p[12] + p[13] - p[14]) + fx / 2.0) * inv;
                    double uy = ((p[3] - p[4] + p[7] + p[8] - p[9] - p[10] + p[15] - p[16] + p[17] - p[18]) + fy / 2.0) * inv;
                    double uz = ((p[5] - p[6] + p[11] + p[12] - p[13] - p[14] + p[15] + p[16] - p[17] - p[18]) + fz / 2.0) * inv;
                    double usq = ux * ux + uy * uy + uz * uz;
                    const double wr = 1.0 / 3.0, wa = 1.0 / 18.0, we = 1.0 / 36.0;
                    const double t3 = 3.0, t45 = 4.5, t15 = 1.5, t9 = 9.0;
                    double gp = 1.0 - omega / 2.0;
                    double feq, S, cu, cf;
#define OR_FEQ(w) ((w) * rho * (1.0 + t3 * cu + t45 * cu * cu - t15 * usq))
#define OR_UPD(q) p[q] = p[q] - omega * (p[q] - feq) + gp * S
                    feq = wr * rho * (1.0 - t15 * usq);
                    S = wr * ((-ux) * fx + (-uy) * fy + (-uz) * fz) * t3; OR_UPD(0);
                    cu = ux; feq = OR_FEQ(wa);
                    S = wa * ((1.0 - ux) * fx + (-uy) * fy + (-uz) * fz) * t3 + wa * cu * fx * t9; OR_UPD(1);
                    cu = -ux; feq = OR_FEQ(wa);
                    S = wa * ((-1.0 - ux) * fx + (-uy) * fy + (-uz) * fz) * t3 + wa * cu * (-fx) * t9; OR_UPD(2);
                    cu = uy; feq = OR_FEQ(wa);
                    S = wa * ((-ux) * fx + (1.0 - uy) * fy + (-uz) * fz) * t3 + wa * cu * fy * t9; OR_UPD(3);
                    cu = -uy; feq = OR_FEQ(wa);
                    S = wa * ((-ux) * fx + (-1.0 - uy) * fy + (-uz) * fz) * t3 + wa * cu * (-fy) * t9; OR_UPD(4);
                    cu = uz; feq = OR_FEQ(wa);
                    S = wa * ((-ux) * fx + (-uy) * fy + (1.0 - uz) * fz) * t3 + wa * cu * fz * t9; OR_UPD(5);
                    cu = -uz; feq = OR_FEQ(wa);
                    S = wa * ((-ux) * fx + (-uy) * fy + (-1.0 - uz) * fz) * t3 + wa * cu * (-fz) * t9; OR_UPD(6);
                    cu = ux + uy; cf = fx + fy; feq = OR_FEQ(we);
                    S = we * ((1.0 - ux) * fx + (1.0 - uy) * fy + (-uz) * fz) * t3 + we * cu * cf * t9; OR_UPD(7);
                    cu = -ux + uy; cf = -fx + fy; feq = OR_FEQ(we);
                    S = we * ((-1.0 - ux) * fx + (1.0 - uy) * fy + (-uz) * fz) * t3 + we * cu * cf * t9; OR_UPD(8);
                    cu = ux - uy; cf = fx - fy; feq = OR_FEQ(we);
                    S = we * ((1.0 - ux) * fx + (-1.0 - uy) * fy + (-uz) * fz) * t3 + we * cu * cf * t9; OR_UPD(9);
                    cu = -ux - uy; cf = -fx - fy; feq = OR_FEQ(we);
                    S = we * ((-1.0 - ux) * fx + (-1.0 - uy) * fy + (-uz) * fz) * t3 + we * cu * cf * t9; OR_UPD(10);
                    cu = ux + uz; cf = fx + fz; feq = OR_FEQ(we);
                    S = we * ((1.0 - ux) * fx + (-uy) * fy + (1.0 - uz) * fz) * t3 + we * cu * cf * t9; OR_UPD(11);
                    cu = -ux + uz; cf = -fx + fz; feq = OR_FEQ(we);
                    S = we * ((-1.0 - ux) * fx + (-uy) * fy + (1.0 - uz) * fz) * t3 + we * cu * cf * t9; OR_UPD(12);
                    cu = ux - uz; cf = fx - fz; feq = OR_FEQ(we);
                    S = we * ((1.0 - ux) * fx + (-uy) * fy + (-1.0 - uz) * fz) * t3 + we * cu * cf * t9; OR_UPD(13);
                    cu = -ux - uz; cf = -fx - fz; feq = OR_FEQ(we);
                    S = we * ((-1.0 - ux) * fx + (-uy) * fy + (-1.0 - uz) * fz) * t3 + we * cu * cf * t9; OR_UPD(14);
                    cu = uy + uz; cf = fy + fz; feq = OR_FEQ(we);
                    S = we * ((-ux) * fx + (1.0 - uy) * fy + (1.0 - uz) * fz) * t3 + we * cu * cf * t9; OR_UPD(15);
                    cu = -uy + uz; cf = -fy + fz; feq = OR_FEQ(we);
                    S = we * ((-ux) * fx + (-1.0 - uy) * fy + (1.0 - uz) * fz) * t3 + we * cu * cf * t9; OR_UPD(16);
                    cu = uy - uz; cf = fy - fz; feq = OR_FEQ(we);
                    S = we * ((-ux) * fx + (1.0 - uy) * fy + (-1.0 - uz) * fz) * t3 + we * cu * cf * t9; OR_UPD(17);
                    cu = -uy - uz; cf = -fy - fz; feq = OR_FEQ(we);
                    S = we * ((-ux) * fx + (-1.0 - uy) * fy + (-1.0 - uz) * fz) * t3 + we * cu * cf * t9; OR_UPD(18);
#undef OR_FEQ
#undef OR_UPD
                }
                for (int q = 0; q < 19; ++q) f[I3(i, j, k, q)] = p[q];
            }
}

/* ------------------------------------------------------------------------ */
/* Interpolated bounce-back: src/kernels/li_bb_2d_v2.jl, li_bb_3d_v2.jl     */
/* ------------------------------------------------------------------------ */

/* _libb_branch: src/kernels/li_bb_2d.jl:70-83 */
static inline double libb_branch(double q_w, double f_here, double f_back, double f_bar_here,
                                 double d) {
    if (q_w <= 0.5) return 2.0 * q_w * f_here + (1.0 - 2.0 * q_w) * f_back + d;
    double inv = 1.0 / (2.0 * q_w);
    return inv * f_here + (1.0 - inv) * f_bar_here + d * inv;
}

/* fused_trt_libb_v2_step!: li_bb_2d_v2.jl:35-41 (PullHalfwayBB, SolidInert,
 * ApplyLiBBPrePhase of dsl/bricks.jl:516-560, Moments, CollideTRTDirect,
 * WriteMoments).  Rates are passed already rounded to the storage type. */
void or_fused_trt_libb_2d(double *f_out, const double *f_in, double *rho_o, double *ux_o,
                          double *uy_o, const uint8_t *solid, const double *qw,
                          const double *uwx, const double *uwy, int Nx, int Ny, double sp,
                          double sm) {
    for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i) {
            size_t n = N2(i, j);
            if (solid && solid[n]) {
                double feq[9];
                feq2d_all(1.0, 0.0, 0.0, 0.0, feq);
                for (int q = 0; q < 9; ++q) f_out[I2(i, j, q)] = feq[q];
                if (rho_o) { rho_o[n] = 1.0; ux_o[n] = 0.0; uy_o[n] = 0.0; }
                continue;
            }
            double p[9];
            pull2d(f_in, Nx, Ny, i, j, p);
#define QW(q) qw[I2(i, j, q)]
#define FI(q) f_in[I2(i, j, q)]
#define UX(q) uwx[I2(i, j, q)]
#define UY(q) uwy[I2(i, j, q)]
            /* reference q 2/4 (east/west), 3/5, 6/8, 7/9 */
            if (QW(1) > 0.0) p[3] = libb_branch(QW(1), FI(1), p[1], FI(3), -(2.0 / 3.0) * UX(1));
            if (QW(3) > 0.0) p[1] = libb_branch(QW(3), FI(3), p[3], FI(1), (2.0 / 3.0) * UX(3));
            if (QW(2) > 0.0) p[4] = libb_branch(QW(2), FI(2), p[2], FI(4), -(2.0 / 3.0) * UY(2));
            if (QW(4) > 0.0) p[2] = libb_branch(QW(4), FI(4), p[4], FI(2), (2.0 / 3.0) * UY(4));
            if (QW(5) > 0.0)
                p[7] = libb_branch(QW(5), FI(5), p[5], FI(7), -(1.0 / 6.0) * (UX(5) + UY(5)));
            if (QW(7) > 0.0)
                p[5] = libb_branch(QW(7), FI(7), p[7], FI(5), (1.0 / 6.0) * (UX(7) + UY(7)));
            if (QW(6) > 0.0)
                p[8] = libb_branch(QW(6), FI(6), p[6], FI(8), -(1.0 / 6.0) * (-UX(6) + UY(6)));
            if (QW(8) > 0.0)
                p[6] = libb_branch(QW(8), FI(8), p[8], FI(6), (1.0 / 6.0) * (-UX(8) + UY(8)));
#undef QW
#undef FI
#undef UX
#undef UY
            double rho, ux, uy;
            trt2d_node(p, sp, sm, &rho, &ux, &uy);
            for (int q = 0; q < 9; ++q) f_out[I2(i, j, q)] = p[q];
            if (rho_o) { rho_o[n] = rho; ux_o[n] = ux; uy_o[n] = uy; }
        }
}

/* fused_trt_libb_v2_step_3d!: li_bb_3d_v2.jl:13-42, ApplyLiBBPrePhase_3D of
 * dsl/bricks_3d.jl:367-475, with the periodic pull of or_fused_trt_3d. */
void or_fused_trt_libb_3d(double *f_out, const double *f_in, double *rho_o, double *ux_o,
                          double *uy_o, double *uz_o, const uint8_t *solid, const double *qw,
                          const double *uwx, const double *uwy, const double *uwz, int Nx,
                          int Ny, int Nz, double sp, double sm, int per_x, int per_y,
                          int per_z) {
    for (int k = 0; k < Nz; ++k)
        for (int j = 0; j < Ny; ++j)
            for (int i = 0; i < Nx; ++i) {
                size_t n = N3(i, j, k);
                double feq[19];
                if (solid && solid[n]) {
                    feq3d_all(1.0, 0.0, 0.0, 0.0, 0.0, feq);
                    for (int q = 0; q < 19; ++q) f_out[I3(i, j, k, q)] = feq[q];
                    if (rho_o) { rho_o[n] = 1.0; ux_o[n] = 0.0; uy_o[n] = 0.0; uz_o[n] = 0.0; }
                    continue;
                }
                double p[19];
                pull3d(f_in, Nx, Ny, Nz, i, j, k, per_x, per_y, per_z, p);
#define QW(q) qw[I3(i, j, k, q)]
#define FI(q) f_in[I3(i, j, k, q)]
#define UX(q) uwx[I3(i, j, k, q)]
#define UY(q) uwy[I3(i, j, k, q)]
#define UZ(q) uwz[I3(i, j, k, q)]
#define LINK(a, b, d) if (QW(a) > 0.0) p[b] = libb_branch(QW(a), FI(a), p[a], FI(b), d)
                const double c3 = 1.0 / 3.0, c6 = 1.0 / 6.0;
                LINK(1, 2, -c3 * UX(1));
                LINK(2, 1, c3 * UX(2));
                LINK(3, 4, -c3 * UY(3));
                LINK(4, 3, c3 * UY(4));
                LINK(5, 6, -c3 * UZ(5));
                LINK(6, 5, c3 * UZ(6));
                LINK(7, 10, -c6 * (UX(7) + UY(7)));
                LINK(10, 7, c6 * (UX(10) + UY(10)));
                LINK(8, 9, -c6 * (-UX(8) + UY(8)));
                LINK(9, 8, -c6 * (UX(9) - UY(9)));
                LINK(11, 14, -c6 * (UX(11) + UZ(11)));
                LINK(14, 11, c6 * (UX(14) + UZ(14)));
                LINK(12, 13, -c6 * (-UX(12) + UZ(12)));
                LINK(13, 12, -c6 * (UX(13) - UZ(13)));
                LINK(15, 18, -c6 * (UY(15) + UZ(15)));
                LINK(18, 15, c6 * (UY(18) + UZ(18)));
                LINK(16, 17, -c6 * (-UY(16) + UZ(16)));
                LINK(17, 16, -c6 * (UY(17) - UZ(17)));
#undef LINK
#undef QW
#undef FI
#undef UX
#undef UY
#undef UZ
                double rho, ux, uy, uz;
                moments3d(p, &rho, &ux, &uy, &uz);
                double usq = ux * ux + uy * uy + uz * uz;
                feq3d_all(rho, ux, uy, uz, usq, feq);
                double a = (sp + sm) * 0.5, b = (sp - sm) * 0.5;
                static const int pa[9] = {1, 3, 5, 7, 8, 11, 12, 15, 16};
                static const int pb[9] = {2, 4, 6, 10, 9, 14, 13, 18, 17};
                f_out[I3(i, j, k, 0)] = p[0] - sp * (p[0] - feq[0]);
                for (int m = 0; m < 9; ++m) {
                    int x = pa[m], y = pb[m];
                    f_out[I3(i, j, k, x)] = p[x] - a * (p[x] - feq[x]) - b * (p[y] - feq[y]);
                    f_out[I3(i, j, k, y)] = p[y] - a * (p[y] - feq[y]) - b * (p[x] - feq[x]);
                }
                if (rho_o) { rho_o[n] = rho; ux_o[n] = ux; uy_o[n] = uy; uz_o[n] = uz; }
            }
}

/* collide_guo_2d! (src/kernels/collide_guo_2d.jl:5-81; Fxf == NULL: constant
 * force) and collide_guo_field_2d! (:93-155, per-node force), population by
 * population as the reference writes them. */
void or_collide_guo_2d(double *f, const uint8_t *solid, const double *Fxf, const double *Fyf,
                       int Nx, int Ny, double omega, double Fx, double Fy) {
    for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i) {
            double p[9];
            size_t n = N2(i, j);
            for (int q = 0; q < 9; ++q) p[q] = f[I2(i, j, q)];
            if (solid && solid[n]) {
                swap_pairs_2d(p);
            } else {
                double fx = Fxf ? Fxf[n] : Fx, fy = Fyf ? Fyf[n] : Fy;
                double rho = p[0] + p[1] + p[2] + p[3] + p[4] + p[5] + p[6] + p[7] + p[8];
                double inv = 1.0 / rho;
                double ux = ((p[1] - p[3] + p[5] - p[6] - p[7] + p[8]) + fx / 2.0) * inv;
                double uy = ((p[2] - p[4] + p[5] + p[6] - p[7] - p[8]) + fy / 2.0) * inv;
                double usq = ux * ux + uy * uy;
                double gp = 1.0 - omega / 2.0, feq[9], S[9];
                feq2d_all(rho, ux, uy, usq, feq);
                S[0] = 4.0 / 9.0 * ((-ux) * fx + (-uy) * fy) * 3.0;
                S[1] = 1.0 / 9.0 * ((1.0 - ux) * fx + (-uy) * fy) * 3.0 + 1.0 / 9.0 * (ux) * (fx) * 9.0;
                S[2] = 1.0 / 9.0 * ((-ux) * fx + (1.0 - uy) * fy) * 3.0 + 1.0 / 9.0 * (uy) * (fy) * 9.0;
                S[3] = 1.0 / 9.0 * ((-1.0 - ux) * fx + (-uy) * fy) * 3.0 + 1.0 / 9.0 * (-ux) * (-fx) * 9.0;
                S[4] = 1.0 / 9.0 * ((-ux) * fx + (-1.0 - uy) * fy) * 3.0 + 1.0 / 9.0 * (-uy) * (-fy) * 9.0;
                S[5] = 1.0 / 36.0 * ((1.0 - ux) * fx + (1.0 - uy) * fy) * 3.0 + 1.0 / 36.0 * (ux + uy) * (fx + fy) * 9.0;
                S[6] = 1.0 / 36.0 * ((-1.0 - ux) * fx + (1.0 - uy) * fy) * 3.0 + 1.0 / 36.0 * (-ux + uy) * (-fx + fy) * 9.0;
                S[7] = 1.0 / 36.0 * ((-1.0 - ux) * fx + (-1.0 - uy) * fy) * 3.0 + 1.0 / 36.0 * (-ux - uy) * (-fx - fy) * 9.0;
                S[8] = 1.0 / 36.0 * ((1.0 - ux) * fx + (-1.0 - uy) * fy) * 3.0 + 1.0 / 36.0 * (ux - uy) * (fx - fy) * 9.0;
                for (int q = 0; q < 9; ++q) p[q] = p[q] - omega * (p[q] - feq[q]) + gp * S[q];
            }
            for (int q = 0; q < 9; ++q) f[I2(i, j, q)] = p[q];
        }
}

/* compute_macroscopic_forced_2d!: src/kernels/macroscopic.jl:84-99 */
void or_macroscopic_forced_2d(double *rho, double *ux, double *uy, const double *f, int Nx, int Ny,
                              double Fx, double Fy) {
    for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i) {
            const double *p[9];
            for (int q = 0; q < 9; ++q) p[q] = &f[I2(i, j, q)];
            double r = *p[0] + *p[1] + *p[2] + *p[3] + *p[4] + *p[5] + *p[6] + *p[7] + *p[8];
            double inv = 1.0 / r;
            rho[N2(i, j)] = r;
            ux[N2(i, j)] = ((*p[1] - *p[3] + *p[5] - *p[6] - *p[7] + *p[8]) + Fx / 2.0) * inv;
            uy[N2(i, j)] = ((*p[2] - *p[4] + *p[5] + *p[6] - *p[7] - *p[8]) + Fy / 2.0) * inv;
        }
}

/* compute_macroscopic_forced_3d! / _field_3d!: src/kernels/macroscopic.jl:121-192
 * (Fxf == NULL: constant force). */
void or_macroscopic_forced_3d(double *rho, double *ux, double *uy, double *uz, const double *f,
                              int Nx, int Ny, int Nz, double Fx, double Fy, double Fz,
                              const double *Fxf, const double *Fyf, const double *Fzf) {
    for (int k = 0; k < Nz; ++k)
        for (int j = 0; j < Ny; ++j)
            for (int i = 0; i < Nx; ++i) {
                double p[19];
                size_t n = N3(i, j, k);
                for (int q = 0; q < 19; ++q) p[q] = f[I3(i, j, k, q)];
                double r = p[0] + p[1] + p[2] + p[3] + p[4] + p[5] + p[6] + p[7] + p[8] + p[9] +
                           p[10] + p[11] + p[12] + p[13] + p[14] + p[15] + p[16] + p[17] + p[18];
                double inv = 1.0 / r;
                double fx = Fxf ? Fxf[n] : Fx, fy = Fyf ? Fyf[n] : Fy, fz = Fzf ? Fzf[n] : Fz;
                rho[n] = r;
                ux[n] = ((p[1] - p[2] + p[7] - p[8] + p[9] - p[10] + p[11] - p[12] + p[13] - p[14]) + fx / 2.0) * inv;
                uy[n] = ((p[3] - p[4] + p[7] + p[8] - p[9] - p[10] + p[15] - p[16] + p[17] - p[18]) + fy / 2.0) * inv;
                uz[n] = ((p[5] - p[6] + p[11] + p[12] - p[13] - p[14] + p[15] + p[16] - p[17] - p[18]) + fz / 2.0) * inv;
            }
}

/* stream_periodic_xz_wall_y_3d!: src/kernels/stream_periodic_3d.jl:24-84 (pull
 * with x and z wrapped, half-way bounce-back at the y faces); the general
 * per-axis form. */
void or_stream_periodic_3d(double *f_out, const double *f_in, int Nx, int Ny, int Nz, int px,
                           int py, int pz) {
    for (int k = 0; k < Nz; ++k)
        for (int j = 0; j < Ny; ++j)
            for (int i = 0; i < Nx; ++i) {
                double fp[19];
                pull3d(f_in, Nx, Ny, Nz, i, j, k, px, py, pz, fp);
                for (int q = 0; q < 19; ++q) f_out[I3(i, j, k, q)] = fp[q];
            }
}
