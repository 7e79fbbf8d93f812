"""Work accounting used for roofline figures (one place, fixed convention).

Flops per interaction, FP32 mixed path, counting add/mul/FMA-as-2/sqrt/rsqrt/
div as 1 each (an FMA counts 2):
  gravity particle-node (monopole + traceless quadrupole)   GRAV_NODE_QUAD
  gravity particle-node (monopole only)                     GRAV_NODE_MONO
  gravity particle-particle with spline softening branch    GRAV_PART
  density (+EOS) pair inside the support                    DENSITY_PAIR
  hydro pair (accel + du/dt + viscosity + Balsara)          HYDRO_PAIR
  h-search candidate (distance + two threshold compares)    H_PAIR
The walk kernels count candidates (every staged source visited by every
target), so achieved flops are a lower bound of the issued work.

Algorithmic HBM bytes per particle per step (compulsory traffic, mixed
path): see BYTES.  Sort/gather/KDK are HBM-bound; walks are FP32-issue bound.
"""

GRAV_NODE_QUAD = 50
GRAV_NODE_MONO = 23
GRAV_PART = 30
DENSITY_PAIR = 20
HYDRO_PAIR = 75
H_PAIR = 8

BYTES = {
    # kick + drift (r, v, a read; r, v written) + key (r read, key/idx written)
    "kick_drift_keys": 72 + 24 + 12,
    # 6 LSD passes of (8 B key + 4 B index): hist read 8, scatter read 12 + write 12
    "sort": 6 * (8 + 12 + 12),
    # 12 FP64 fields + orig gathered (read + write) + 3 float4 packs written
    "gather": 2 * (12 * 8 + 8) + 3 * 16,
    "tree": 15,
    "h": 40,
    "density": 40,
    "gravity": 40,
    "hydro": 72,
    # u update (u, u_prev, dudt, dudt_prev read; u, u_prev, dudt_prev written)
    # + second kick (a_g, a_sph, v read; a, v, packed v written)
    "kick_u": 56 + 136,
}
