// validate.h - argument checks of a grid and parameter set, shared by
// bolt_ctx_create and bolt_dfdt_noalloc (the reference raises the matching
// Python exceptions in physical_system.py:77-144 and boundaries.py:415-577).
#pragma once

#include "../../include/bolt_b200.h"

namespace bolt {

inline bool bc_is_mirror(int bc) { return bc == BOLT_BC_MIRROR || bc == BOLT_BC_MIRROR_DIRICHLET; }

// BOLT_OK, BOLT_ERR_ARG (out of range) or BOLT_ERR_UNSUPPORTED (a valid
// combination this build has no kernel for)
inline int check_grid_params(const BoltGrid& g, const BoltParams& p) {
    if (g.N_q1 < 1 || g.N_q2 < 1 || g.N_p1 < 1 || g.N_p2 < 1 || g.N_p3 < 1 || g.N_ghost < 0 ||
        g.N_s < 1 || g.N_s > BOLT_MAX_SPECIES)
        return BOLT_ERR_ARG;
    if (p.dtype != BOLT_F64 && p.dtype != BOLT_F32 && p.dtype != BOLT_F64_FAST)
        return BOLT_ERR_ARG;
    if (p.recon_q < 0 || p.recon_q > 3 || p.recon_p < 0 || p.recon_p > 3) return BOLT_ERR_ARG;
    if (p.integrator != BOLT_RK2 && p.integrator != BOLT_RK4) return BOLT_ERR_ARG;
    if (p.p_dim < 1 || p.p_dim > 3) return BOLT_ERR_ARG;
    if (p.bc_q1 < BOLT_BC_PERIODIC || p.bc_q1 > BOLT_BC_SHEARING_BOX ||
        p.bc_q2 < BOLT_BC_PERIODIC || p.bc_q2 > BOLT_BC_SHEARING_BOX)
        return BOLT_ERR_ARG;
    // shearing box: one axis, the other periodic, a 4-point stencil in the strip
    if (p.bc_q1 == BOLT_BC_SHEARING_BOX || p.bc_q2 == BOLT_BC_SHEARING_BOX) {
        const int other = p.bc_q1 == BOLT_BC_SHEARING_BOX ? p.bc_q2 : p.bc_q1;
        if (other != BOLT_BC_PERIODIC || g.N_ghost < 2) return BOLT_ERR_UNSUPPORTED;
    }
    // fields: periodic axes, or a block's external cuts (electrodynamic only:
    // the FFT solve is serial, fft.py:26-27)
    if (p.fields_enabled) {
        for (int bc : {p.bc_q1, p.bc_q2}) {
            if (bc == BOLT_BC_PERIODIC) continue;
            if (bc == BOLT_BC_EXTERNAL && p.fields_type == BOLT_FIELDS_ELECTRODYNAMIC) continue;
            return BOLT_ERR_UNSUPPORTED;
        }
    }
    if (p.fields_enabled && p.fields_type != BOLT_FIELDS_ELECTRODYNAMIC &&
        p.fields_type != BOLT_FIELDS_ELECTROSTATIC)
        return BOLT_ERR_ARG;
    if (g.N_ghost == 0 && (p.bc_q1 != BOLT_BC_PERIODIC || p.bc_q2 != BOLT_BC_PERIODIC))
        return BOLT_ERR_UNSUPPORTED;
    // a mirror image of the ghost zone must lie inside the grid
    if ((bc_is_mirror(p.bc_q1) && g.N_ghost > g.N_q1) ||
        (bc_is_mirror(p.bc_q2) && g.N_ghost > g.N_q2))
        return BOLT_ERR_UNSUPPORTED;
    return BOLT_OK;
}

}  // namespace bolt
