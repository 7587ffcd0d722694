// The ray march of the synthetic tomography builder, shared by its host and
// device versions (qb_synth.cpp, qb_synth_gpu.cu).
#pragma once

#include <cstdint>
#include <vector>

#include "qublar.h"

namespace qb {

struct Grid {
    double lo[3];
    double v;
    int n[3];
    int64_t cells() const { return int64_t(n[0]) * n[1] * n[2]; }
};

// One sky bin after the march: optical depths through the pyramid (tau0 all
// rock, tau with the void) and its entries [first, first + cnt) in the flat
// lists, bits in the order the sub-rays first reach them.
struct BinMarch {
    double tau0 = 0.0, tau = 0.0;
    int64_t first = 0, cnt = 0;
};

// Everything the march reads. Sky bin (k, it, ip) is bin (k n_theta + it)
// n_phi + ip; its sub-ray (su, sv) has direction (sth cph, sth sph, cth) with
// cth / sth = cos / sin of the zenith angle at [it S + su] and cph / sph =
// cos / sin of the azimuth at [(k n_phi + ip) S + sv].
struct SynthMarch {
    Grid g;
    std::vector<uint8_t> rock, is_void;   // per cell
    std::vector<int32_t> cell_bit;        // per cell: its bit, or -1
    int n_det = 0;
    double det[12] = {};
    int n_theta = 0, n_phi = 0, S = 1, n_bits = 0;
    double inv_s2 = 1.0, mu_rock = 0.0, mu_air = 0.0;
    std::vector<double> cth, sth, cph, sph;
};

// The device march: the same bins, entries and depths as the host's, bit for
// bit; QB_ENOTSUP when a bin reaches more bits than the device lists hold.
qb_status synth_march_device(const SynthMarch& M, const qb_opts* opts, std::vector<BinMarch>& bins,
                             std::vector<int32_t>& e_bit, std::vector<float>& e_a);

}  // namespace qb
