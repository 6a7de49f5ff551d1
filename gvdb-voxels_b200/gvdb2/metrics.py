"""Algorithmic HBM bytes of the point -> sparse-volume step.

Each array is counted once at its natural width; sort passes, scratch and
re-reads are overhead and not counted.  Symbols:
  N  points, P = 12 position bytes, Cw point-attribute floats scattered,
  G  gathered floats per point, C grid channels written by the scatter,
  Cg grid channels read by the gather, B active bricks, T tile voxels incl.
  apron, R3 interior voxels per brick, U unique nodes (all levels),
  CL child-list bytes of the interior nodes.
"""

P_BYTES = 12


def stage_bytes(N, B, U, C, Cw, G, T, R3, CL=0, Cg=None):
    Cg = G if Cg is None else Cg
    return {
        "topology": P_BYTES * N + 4 * N + 8 * U + 64 * U + CL,
        "binning": 4 * N + 4 * N,
        "scatter": P_BYTES * N + 4 * Cw * N + 4 * N + 4 * C * B * T,
        "apron": 2 * 4 * C * B * (T - R3),
        "gather": P_BYTES * N + 4 * N + 4 * G * N + 4 * Cg * B * T,
    }


def step_bytes(**kw):
    return sum(stage_bytes(**kw).values())


def adjoint_bytes(N, B, C, Cw, T):
    """Extra bytes of the adjoint: grad-grid read plus per-point grad writes."""
    return 4 * C * B * T + (P_BYTES + 4 * Cw) * N
