"""CPU restatement of the learned thin boundary's arithmetic (TEST INFRASTRUCTURE ONLY).

It restates, in numpy, what the device code of cmakepro_cuda_seissim_v2_b200/csrc/
seis3d_boundary.cuh computes, so that the tests can check the kernels against it:

* the boundary columns of each CPML face and their inputs (8-cell stencil of the nine fields
  along the face normal, lateral central differences, the six CPML memories of the face's
  axis on the 4 CPML cells, RMS amplitude s, impedance scaling of the stresses, five scheme
  numbers), and the corrected-cell ownership rule;
* the network's forward pass and the gradient of the weighted squared error, with BF16
  rounding (round to nearest even) at the same points as the tensor-core kernels: inputs,
  weights, both hidden activations, dL/dy and both hidden-layer gradients before they enter
  a product; every product accumulates in FP64 here (FP32 on the device).

The network has no counterpart in the reference (its CPML is 8-40 cells and has no learned
part); the scheme numbers it reads follow the reference's definitions (Courant number
v dt / h, CPML profile of cuda/Cuda_Seis3D.cu:44-64).
"""
from __future__ import annotations

import numpy as np

IN, HIDDEN, OUT, OUT_PAD = 256, 64, 36, 48
SCHEME = 240   # first scheme input (216 field inputs, 24 CPML memories before it)
W1, W2, W3 = 0, HIDDEN * IN, HIDDEN * IN + HIDDEN * HIDDEN
MATRICES = W3 + OUT_PAD * HIDDEN
B1, B2, B3 = MATRICES, MATRICES + HIDDEN, MATRICES + 2 * HIDDEN
PARAMETERS = B3 + OUT_PAD
FACES = 6
LATERAL = {0: (1, 2), 1: (0, 2), 2: (0, 1)}   # normal axis -> lateral axes (x = 0, y = 1, z = 2)


def bf16(x) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest, ties to even), returned as float32."""
    b = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32)


def unpack(params: np.ndarray):
    p = np.asarray(params, dtype=np.float32)
    return (p[W1:W2].reshape(HIDDEN, IN), p[W2:W3].reshape(HIDDEN, HIDDEN), p[W3:MATRICES].reshape(OUT_PAD, HIDDEN),
            p[B1:B2], p[B2:B3], p[B3:PARAMETERS])


def forward(params, x):
    """Outputs (rows x 48, normalised units) and the BF16 hidden activations."""
    w1, w2, w3, b1, b2, b3 = unpack(params)
    xb = bf16(x).astype(np.float64)
    h1 = bf16(np.maximum(xb @ bf16(w1).astype(np.float64).T + b1, 0)).astype(np.float64)
    h2 = bf16(np.maximum(h1 @ bf16(w2).astype(np.float64).T + b2, 0)).astype(np.float64)
    y = h2 @ bf16(w3).astype(np.float64).T + b3
    return y, xb, h1, h2


def gradients(params, x, t, w, out_scale):
    """Gradient of sum_rows w (y - t / out_scale)^2 over the parameters, and that sum."""
    w1, w2, w3, b1, b2, b3 = unpack(params)
    y, xb, h1, h2 = forward(params, x)
    target = np.zeros((len(x), OUT_PAD))
    target[:, :OUT] = np.asarray(t, dtype=np.float64) / out_scale
    diff = y - target
    diff[:, OUT:] = 0.0
    wcol = np.asarray(w, dtype=np.float64)[:, None]
    loss = float(np.sum(wcol * diff * diff))
    dy = 2.0 * wcol * diff
    dyb = bf16(dy.astype(np.float32)).astype(np.float64)
    dz2 = (dyb @ bf16(w3).astype(np.float64)) * (h2 > 0)
    dz2b = bf16(dz2.astype(np.float32)).astype(np.float64)
    dz1 = (dz2b @ bf16(w2).astype(np.float64)) * (h1 > 0)
    dz1b = bf16(dz1.astype(np.float32)).astype(np.float64)
    g = np.zeros(PARAMETERS)
    g[W1:W2] = (dz1b.T @ xb).ravel()
    g[W2:W3] = (dz2b.T @ h1).ravel()
    gw3 = dyb.T @ h2
    gw3[OUT:] = 0.0
    g[W3:MATRICES] = gw3.ravel()
    g[B1:B2] = dz1.sum(0)
    g[B2:B3] = dz2.sum(0)
    gb3 = dy.sum(0)
    gb3[OUT:] = 0.0
    g[B3:PARAMETERS] = gb3
    return g, loss


def faces(context):
    """Present CPML faces: index -> (normal axis, side, lateral extents, owning faces of the
    lateral ends)."""
    c = context
    present = [not c.reflecting3D and not (f == 4 and c.freeSurface3D) for f in range(FACES)]
    n = (c.nx3D, c.ny3D, c.nz3D)
    out = {}
    for f in range(FACES):
        if not present[f]:
            continue
        axis, side = divmod(f, 2)
        ua, wa = LATERAL[axis]
        ends = [2 * ua if present[2 * ua] else -1, 2 * ua + 1 if present[2 * ua + 1] else -1,
                2 * wa if present[2 * wa] else -1, 2 * wa + 1 if present[2 * wa + 1] else -1]
        out[f] = (axis, side, n[ua], n[wa], ends)
    return out


def cell(context, face, u, w, d):
    """Grid (x, y, z) of stencil cell d (0..3 interior deepest first, 4..7 CPML) of column (u, w)."""
    c = context
    axis, side = divmod(face, 2)
    ua, wa = LATERAL[axis]
    o = (c.ox3D, c.oy3D, c.oz3D)
    n = (c.nx3D, c.ny3D, c.nz3D)
    p = [0, 0, 0]
    p[ua] = o[ua] + u
    p[wa] = o[wa] + w
    edge = o[axis] + n[axis] - 1 if side else o[axis]
    p[axis] = edge + (d - 3) * (1 if side else -1)
    return tuple(p)


def owns(face, nu, nw, ends, u, w, d):
    depth = 3 - d
    for e, dist in zip(ends, (u, nu - 1 - u, w, nw - 1 - w)):
        if e < 0 or dist >= 4:
            continue
        if dist < depth or (dist == depth and e < face):
            return False
    return True


def psi_value(context, psi, pitch, axis, slot, x, y, z):
    """CPML memory `slot` of axis `axis` at grid cell (x, y, z), from the session's slab arrays
    (flat host copies): x slab [slot][z][y][q], y slab [slot][z][q][x pitched], z slab
    [slot][q][y][x pitched]; q counts slab cells from the low end."""
    c = context
    p = c.pml3D
    top_free = axis == 2 and c.freeSurface3D
    n = (c.gx3D, c.gy3D, c.gz3D)[axis]
    coord = (x, y, z)[axis]
    if not top_free and coord < 4 + p:
        q = coord - 4
    else:
        q = (0 if top_free else p) + coord - (n - 4 - p)
    thick = (1 if top_free else 2) * p
    if axis == 0:
        return float(psi[0][slot * c.gz3D * c.gy3D * 2 * p + (z * c.gy3D + y) * 2 * p + q])
    if axis == 1:
        return float(psi[1][slot * c.gz3D * 2 * p * pitch + (z * 2 * p + q) * pitch + x])
    return float(psi[2][slot * thick * c.gy3D * pitch + (q * c.gy3D + y) * pitch + x])


def column_inputs(context, fields, materials, face, u, w, psi, pitch):
    """(inputs[256] before BF16 rounding, s, impedance) of one column; fields and materials
    are [gz][gy][gx] arrays (9 fields; 1/rho, lambda, mu), psi the three slab arrays."""
    c = context
    axis, _ = divmod(face, 2)
    ua, wa = LATERAL[axis]
    x, y, z = cell(context, face, u, w, 3)
    inv_rho, lam, mu = (float(m[z, y, x]) for m in materials)
    modulus = lam + 2.0 * mu
    imp = np.sqrt(modulus / inv_rho)
    dt_h = float(np.float32(c.dt3D)) / float(np.float32(c.spacing3D))
    cp = np.sqrt(modulus * inv_rho) * dt_h
    cs = np.sqrt(mu * inv_rho) * dt_h
    centre = np.zeros(72)
    du = np.zeros(72)
    dw = np.zeros(72)
    for k in range(9):
        scale = 1.0 if k < 3 else 1.0 / imp
        for d in range(8):
            p = cell(context, face, u, w, d)
            centre[8 * k + d] = fields[k][p[2], p[1], p[0]] * scale
            for arr, lat in ((du, ua), (dw, wa)):
                hi = list(p)
                lo = list(p)
                hi[lat] += 1
                lo[lat] -= 1
                arr[8 * k + d] = (fields[k][hi[2], hi[1], hi[0]] - fields[k][lo[2], lo[1], lo[0]]) * scale
    s = np.sqrt(np.sum(centre ** 2) / 72.0)
    inv = 1.0 / s if s > 0 else 0.0
    x_in = np.zeros(IN)
    x_in[:72] = centre * inv
    x_in[72:144] = du * inv
    x_in[144:216] = dw * inv
    h = float(np.float32(c.spacing3D))
    for slot in range(6):
        for d in range(4):
            q = cell(context, face, u, w, 4 + d)
            x_in[216 + 4 * slot + d] = psi_value(c, psi, pitch, axis, slot, *q) * (h / imp if slot < 3 else h) * inv
    x_in[SCHEME:SCHEME + 5] = [cp, cs, c.maxVp3D * dt_h, c.frequency3D * c.dt3D, 1.0]
    return x_in, s, imp


def corrections(context, fields, materials, psi, pitch, params_by_face, out_scales, gain=1.0):
    """The correction the attached networks add to each field after a step: a dict
    field -> [gz][gy][gx] array (zero outside the owned band cells)."""
    out = [np.zeros_like(np.asarray(f, dtype=np.float64)) for f in fields]
    for face, (axis, side, nu, nw, ends) in faces(context).items():
        rows, where = [], []
        for w in range(nw):
            for u in range(nu):
                x_in, s, imp = column_inputs(context, fields, materials, face, u, w, psi, pitch)
                rows.append(x_in)
                where.append((u, w, s, imp))
        y, *_ = forward(params_by_face[face], np.array(rows, dtype=np.float32))
        for (u, w, s, imp), yr in zip(where, y):
            for k in range(9):
                for d in range(4):
                    if not owns(face, nu, nw, ends, u, w, d):
                        continue
                    x, yy, z = cell(context, face, u, w, d)
                    v = yr[4 * k + d] * out_scales[face] * s * (1.0 if k < 3 else imp)
                    out[k][z, yy, x] += gain * v
    return out
