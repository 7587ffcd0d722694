/*
 * qublar_synth.h -- deterministic synthetic inputs for the annealer.
 *
 * These builders make the QUBOs the solver is measured on. They are input
 * makers, not part of the solve: a caller of the solver brings its own
 * problem. The tomography builder plays the role of the reference's problem
 * builder (build_binary_problem, src/ising_recon.hpp:52-62: BitField::grid,
 * muon_rows and assemble, src/engine.hpp:61-149, src/op_muon.hpp:22-51) on a
 * synthetic pyramid with known truth.
 */
#ifndef QUBLAR_SYNTH_H
#define QUBLAR_SYNTH_H

#include <stdint.h>

#include "qublar.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Muon-tomography QUBO of a square-base pyramid. Units: metres, 1/m. */
typedef struct qb_tomo_params {
    int32_t target_bits;     /* keep this many pyramid cells (x-fastest order); 0 = all */
    int32_t target_rays;     /* keep this many rays (most-counted first); 0 = all */
    double voxel;            /* cube side */
    double half_base;        /* pyramid half base */
    double height;           /* pyramid height */
    int32_t n_detectors;     /* 1..4 point detectors */
    double det[12];          /* detector positions (x, y, z), below the base: z < 0 */
    int32_t n_theta;         /* zenith bins per detector */
    int32_t n_phi;           /* azimuth bins per detector */
    double theta_min;        /* zenith range, radians */
    double theta_max;
    double phi_half;         /* azimuth half-window around the direction to the axis, radians (pi = all) */
    int32_t sub_rays;        /* chords of a bin are averaged over sub_rays^2 sub-rays (1 = centre line) */
    double room_radius;      /* cells closer than this to a detector carry no bit (its room) */
    double mu_rock;          /* rock attenuation */
    double void_center[3];   /* cubic void of air with known truth */
    double void_side;
    double exposure;         /* expected open-sky muons of a vertical bin */
    double min_open;         /* rays with fewer open muons are dropped (op_muon.hpp:30) */
    double lambda;           /* prior: unlike-neighbour cost */
    double kappa;            /* prior: cost of a 1-bit */
    uint64_t seed;           /* Poisson counts */
} qb_tomo_params;

/* The 306,328-bit, 75,594-ray pyramid of the tomography benchmark. */
void qb_tomo_params_default(qb_tomo_params* p);

typedef struct qb_tomo qb_tomo;

qb_status qb_synth_tomography(const qb_tomo_params* p, qb_tomo** out);
/* The same builder with the ray march on the device (one thread per sky bin;
 * opts picks the device and stream, may be NULL): the bits, rays, entries,
 * coefficients and counts equal qb_synth_tomography's bit for bit. The march
 * is the reference builder's O(rays x path) step (muon_rows,
 * src/op_muon.hpp:22-51; the exposure walk of src/muon.cuh:66-134); the
 * Poisson draws and the ray selection stay on the host. QB_ENOTSUP when a sky
 * bin reaches more than 512 bits (qb_synth_tomography builds those). */
qb_status qb_synth_tomography_device(const qb_tomo_params* p, const qb_opts* opts, qb_tomo** out);
/* Sizes: bits, rays, bit-ray entries, neighbour entries. */
qb_status qb_tomo_sizes(const qb_tomo* t, int32_t* n_vars, int32_t* n_rays, int64_t* nnz, int64_t* n_nbr);
/* Copy the problem into caller arrays sized by qb_tomo_sizes; truth (n_vars
 * bytes, 1 = the cell lies in the void) may be NULL. */
qb_status qb_tomo_arrays(const qb_tomo* t, double* d, double* w, int32_t* row_ptr, int32_t* ray, float* a,
                         int32_t* nbr_ptr, int32_t* nbr, uint8_t* truth);
/* The voxel grid (dims: nx, ny, nz; cells x fastest) and the cell of every
 * bit (n_vars entries); either may be NULL. The bits are the grid's domain
 * cells in cell order, as BitField::grid numbers them (src/engine.hpp:61-85). */
qb_status qb_tomo_cells(const qb_tomo* t, int32_t* dims, int64_t* bit_cell);
/* The problem as a descriptor over the builder's own arrays (valid until destroy). */
qb_status qb_tomo_desc(const qb_tomo* t, qb_residual_desc* desc);
void qb_tomo_destroy(qb_tomo* t);

#ifdef __cplusplus
}
#endif

#endif /* QUBLAR_SYNTH_H */
