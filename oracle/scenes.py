"""Seeded synthetic scenes built on the oracle side — TEST INFRASTRUCTURE ONLY.

The inputs of the CPU reference path (the embedded Hex27 hollow cylinder of the
Newton-step benchmark, the Schwarz subdomain choice, the initial state), built
from the oracle's own mesh pipeline (procedural hex box, Hex27 refinement and
keep_cells, restated from fenris/src/mesh/procedural.rs:191-250,
fenris/src/mesh/mesh_convert.rs:163-567 and fenris/src/embedding/mod.rs:291-313
in hoefem_oracle.cpp) and a numpy / libm restatement of the synthetic parts, so
that the reference arm of the benchmark runs without the product library.
`tests/test_oracle_scenes.py` checks every array against the product's scene
generator bit for bit.

Synthetic parts (no reference counterpart; the reference's paper meshes are not
in its repository):
  * cut-cell volume fraction of a background cell: 8 x 8 x 8 midpoint samples of
    the annulus r_in <= r <= r_out around the axis (0.5, 0.5, z); cells with
    phi >= 0.999 are interior, 1e-4 <= phi < 0.999 interface, the rest removed
    (thresholds of fenris/src/embedding/embedding3d.rs:129-143); the volume
    fraction a cut cell reports (the Schwarz rule's input) is its rule's
    embedded volume over the cell volume, as the reference computes it;
  * interface quadrature: per cell Q ~ U{q_min..q_max} points uniform in the
    reference cell [-1, 1]^3 and Dirichlet(1, ..., 1) weights summing to
    8 phi (exponential draws normalised);
  * interior cells: hex_quadrature_strength_5 (fenris/src/quadrature.rs), read
    from the golden fixture extracted from the reference's source;
  * Schwarz subdomains: interface cells with phi <= 0.5, every node outside them
    untreated (SchwarzPreconditionerComponent::from_embedded_model,
    simulation_toolbox/src/fem/schwarz_precond.rs:65-127);
  * random numbers: splitmix64, uniforms (z >> 11) 2^-53, Box-Muller normals.
"""
import json
import math
import os

import numpy as np

from . import oracle as O

_GOLDEN = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tests", "golden",
                       "reference_vectors.json")
_GAMMA = 0x9E3779B97F4A7C15
_M64 = (1 << 64) - 1


class SplitMix64:
    """splitmix64 stream (sequential draws, Python integers)."""

    def __init__(self, seed):
        self.s = int(seed) & _M64

    def next(self):
        self.s = (self.s + _GAMMA) & _M64
        z = self.s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
        return z ^ (z >> 31)

    def uniform01(self):
        return float(self.next() >> 11) * (1.0 / 9007199254740992.0)


def random_normal(seed, n, sigma):
    """n samples of N(0, sigma^2): Box-Muller on pairs of splitmix64 uniforms
    (u1 = 1 - U in (0, 1], u2 = U), cos then sin."""
    rng = SplitMix64(seed)
    out = np.zeros(n)
    two_pi = 6.283185307179586476925286766559
    for i in range(0, n, 2):
        u1 = 1.0 - rng.uniform01()
        u2 = rng.uniform01()
        r = math.sqrt(-2.0 * math.log(u1))
        out[i] = sigma * r * math.cos(two_pi * u2)
        if i + 1 < n:
            out[i + 1] = sigma * r * math.sin(two_pi * u2)
    return out


def hex_quadrature_strength_5():
    q = json.load(open(_GOLDEN))["quadrature"]["hex_quadrature_strength_5"]
    return np.array(q["weights"], dtype=np.float64), np.array(q["points"], dtype=np.float64)


class CylinderScene:
    """Arrays of the embedded hollow-cylinder scene."""

    def __init__(self, vertices, interior_conn, interface_conn, interior_rule, iface_offsets, iface_weights,
                 iface_points, volume_fractions, cell_size):
        self.vertices = vertices
        self.interior_conn = interior_conn
        self.interface_conn = interface_conn
        self.interior_rule = interior_rule
        self.iface_offsets = iface_offsets
        self.iface_weights = iface_weights
        self.iface_points = iface_points
        self.volume_fractions = volume_fractions
        self.cell_size = cell_size

    def nodes_below(self, axis, value):
        return np.nonzero(self.vertices[:, axis] <= value)[0].astype(np.int64)

    def schwarz_subdomains(self, threshold=0.5):
        """(subdomain node lists, untreated nodes) of the reference rule."""
        sel = [self.interface_conn[i] for i in range(self.interface_conn.shape[0])
               if self.volume_fractions[i] <= threshold]
        covered = np.zeros(self.vertices.shape[0], dtype=bool)
        for s in sel:
            covered[s] = True
        return sel, np.nonzero(~covered)[0].astype(np.int64)


_HEX8_CORNERS = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                          [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], dtype=np.float64)


def hex8_detj(Xc, xi):
    """det of the trilinear map's Jacobian at reference points xi (k x 3) for
    corner coordinates Xc (k x 8 x 3), vectorised over k with the operation
    order of a scalar loop over the corners (fenris/src/element.rs:1122-1195)."""
    J = np.zeros((xi.shape[0], 9))
    for c in range(8):
        h = _HEX8_CORNERS[c]
        l0 = (1.0 + h[0] * xi[:, 0]) / 2.0
        l1 = (1.0 + h[1] * xi[:, 1]) / 2.0
        l2 = (1.0 + h[2] * xi[:, 2]) / 2.0
        g = (h[0] / 2.0 * l1 * l2, l0 * h[1] / 2.0 * l2, l0 * l1 * h[2] / 2.0)
        for i in range(3):
            for j in range(3):
                J[:, 3 * i + j] += Xc[:, c, i] * g[j]
    return (J[:, 0] * (J[:, 4] * J[:, 8] - J[:, 7] * J[:, 5]) - J[:, 1] * (J[:, 3] * J[:, 8] - J[:, 6] * J[:, 5])
            + J[:, 2] * (J[:, 3] * J[:, 7] - J[:, 6] * J[:, 4]))


def interface_volume_fractions(vertices, conn, offsets, weights, points):
    """Embedded volume of each cut cell (its rule integrated with |det J|
    over the reference cell) divided by the cell's volume (2 x 2 x 2 Gauss)."""
    ne = conn.shape[0]
    counts = np.diff(offsets)
    Xq = vertices[conn[:, :8]][np.repeat(np.arange(ne), counts)]
    dq = hex8_detj(Xq, points)
    g = 1.0 / math.sqrt(3.0)
    gp = np.array([[g if (a & 1) else -g, g if (a & 2) else -g, g if (a & 4) else -g] for a in range(8)])
    dv = hex8_detj(np.repeat(vertices[conn[:, :8]], 8, axis=0), np.tile(gp, (ne, 1))).reshape(ne, 8)
    out = np.zeros(ne)
    for e in range(ne):
        emb = 0.0
        for q in range(offsets[e], offsets[e + 1]):
            emb += weights[q] * dq[q]
        vol = 0.0
        for a in range(8):
            vol += abs(dv[e, a])
        out[e] = emb / vol
    return out


def embedded_cylinder(n=24, r_inner=0.3, r_outer=0.4, q_min=8, q_max=27, seed=2):
    hx = O.hex_box(1.0, 1, 1, 1, n)
    h27 = O.hex27_from_hex(hx)
    S = 8
    X, C = hx.vertices, hx.cells
    lo, hi = X[C[:, 0]], X[C[:, 6]]
    # x_a = lo + (hi - lo) (a + 0.5) / S, the same operations as a scalar loop
    xs = lo[:, 0:1] + (hi[:, 0:1] - lo[:, 0:1]) * (np.arange(S) + 0.5)[None, :] / S
    ys = lo[:, 1:2] + (hi[:, 1:2] - lo[:, 1:2]) * (np.arange(S) + 0.5)[None, :] / S
    dx = xs - 0.5
    dy = ys - 0.5
    r = np.sqrt(dx[:, :, None] * dx[:, :, None] + dy[:, None, :] * dy[:, None, :])
    inside2 = ((r >= r_inner) & (r <= r_outer)).sum(axis=(1, 2))
    phi = (inside2 * S).astype(np.float64) / float(S * S * S)
    interior = np.nonzero(phi >= 0.999)[0]
    interface = np.nonzero((phi < 0.999) & (phi >= 1e-4))[0]
    keep = np.concatenate([interior, interface]).astype(np.int64)
    km = O.keep_cells(h27, keep)
    ni = interior.size
    rng = SplitMix64(seed)
    offs = [0]
    w_all, p_all = [], []
    for c in interface:
        Q = q_min + int(rng.next() % (q_max - q_min + 1))
        f = float(phi[c])
        e = []
        tot = 0.0
        for _ in range(Q):
            p_all.append((2.0 * rng.uniform01() - 1.0, 2.0 * rng.uniform01() - 1.0, 2.0 * rng.uniform01() - 1.0))
            ev = -math.log(1.0 - rng.uniform01())
            e.append(ev)
            tot += ev
        for ev in e:
            w_all.append(ev / tot * 8.0 * f)
        offs.append(offs[-1] + Q)
    V, fc = km.vertices.copy(), km.cells[ni:].copy()
    offs, w_all, p_all = np.array(offs, dtype=np.int64), np.array(w_all), np.array(p_all).reshape(-1, 3)
    return CylinderScene(V, km.cells[:ni].copy(), fc, hex_quadrature_strength_5(), offs, w_all, p_all,
                         interface_volume_fractions(V, fc, offs, w_all, p_all), 1.0 / n)


def sway_state(scene, amp_x, amp_y, noise_seed):
    """u = (amp_x z^2, amp_y z^2, 0) + N(0, (0.001 h)^2) per DOF, v = 0."""
    X = scene.vertices
    u0 = np.zeros_like(X)
    u0[:, 0] = amp_x * X[:, 2] ** 2
    u0[:, 1] = amp_y * X[:, 2] ** 2
    nd = X.size
    return u0.reshape(-1) + random_normal(noise_seed, nd, 0.001 * scene.cell_size), np.zeros(nd)


def cylinder_reference_scene(scene, young=5e5, poisson=0.45, density=1000.0, cg_tol=1e-6, cg_max_iter=500,
                             threshold=0.5):
    """The oracle Scene of the benchmark step (StVK, bottom nodes fixed,
    gravity, Schwarz subdomains of the reference rule)."""
    ref = O.Scene(scene.vertices)
    w, p = scene.interior_rule
    ref.add_block(O.ELEM_HEX27, scene.interior_conn, w, p)
    ref.add_block(O.ELEM_HEX27, scene.interface_conn, scene.iface_weights, scene.iface_points,
                  qoff=scene.iface_offsets)
    ref.finalize_pattern()
    mu, lam = O.lame(young, poisson)
    ref.set_material(O.MAT_STVK, mu, lam, density)
    ref.set_bc(scene.nodes_below(2, 1e-9))
    ref.set_gravity(True)
    subs, untreated = scene.schwarz_subdomains(threshold)
    ref.set_schwarz(subs, untreated)
    ref.set_solver(cg_tol, cg_max_iter, 100)
    ref.setup()
    return ref
