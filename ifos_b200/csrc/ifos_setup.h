// Host-side set-up of the propagation path: FD coefficients, CPML profiles and
// the per-cell coefficient planes of one model.  All arithmetic follows the
// float/double promotions of the reference's set-up code so that the device
// path starts from bit-identical coefficients.
#pragma once
#include <vector>

#include "ifos_gpu.h"

namespace ifos {

// FD weights hc[0..6] for FDORDER and MAXRELERROR (src/holbergcoeff.c:37-108).
bool fd_coefficients(int fdorder, int maxrelerror, float hc[7]);

// CPML profiles (src/PML_pro.c:83-316): 12 arrays of 2*FW+1 floats, 1-based,
// in the order K_x a_x b_x K_x_half a_x_half b_x_half K_y a_y b_y K_y_half
// a_y_half b_y_half.
struct CpmlProfiles {
    int n = 0;  // 2*FW
    std::vector<float> arr[12];
};
CpmlProfiles cpml_profiles(const ifos_params &p);

// Per-cell coefficient planes of one model, each NY*NX (x fastest).
struct ModelPlanes {
    // common
    std::vector<float> rho, vp, vs, rip, rjp;
    // elastic P-SV / SH
    std::vector<float> uipjp, f_el, g_el;
    // acoustic: g = rho*vp^2
    std::vector<float> g_ac;
    // viscoelastic (src/prepare_update_s.c:50-60)
    std::vector<float> fipjp_v, f_v, g_v, mu_r, pi_r, muipjp_r, taus, taup, tausipjp;
    bool tau_uniform = true;
    float taus0 = 0, taup0 = 0, tausipjp0 = 0;
    // correlation denominators (src/IFOS2D.c:2395-2404): mm = muss*muss (0 where vs<=0),
    // ll = (lamss+muss)^2 in float as the reference evaluates them
    std::vector<float> mm, ll;
    // free-surface row j=1 (src/surface_elastic_PML.c:91-104, src/surface_PML.c:127-147)
    std::vector<float> srf_fjm, srf_g, srf_djm, srf_e;
};

struct ViscoScalars {
    float eta[IFOS_MAX_L + 1];
    float bip[IFOS_MAX_L + 1], bjm[IFOS_MAX_L + 1], cip[IFOS_MAX_L + 1], cjm[IFOS_MAX_L + 1];
    float bjm_srf[IFOS_MAX_L + 1];  // eta/(1+eta/2) of the surface memory update
    float sumu = 0, sumpi = 0;
};
ViscoScalars visco_scalars(const ifos_params &p);

// Builds every plane the physics of `p` needs; returns false on bad input.
bool build_model(const ifos_params &p, const float *vp, const float *vs, const float *rho, const float *taup,
                 const float *taus, ModelPlanes &out);

}  // namespace ifos
