"""A numpy emulation of slab_filter_wide_kernel's data flow, checked against the oracle's apply.

It follows the kernel tile by tile and plane by plane (csrc/filter.cu):
- a CTA owns rows y0 .. y0+TY-1 and columns z0 .. z0+TZ-1 of one lane (TY x TZ = 8 x 32, 8 x 36
  or 13 x 24), and marches x planes q0 .. xe+7 of its chunk (a chunk starting at plane 0 skips the
  7 planes before it);
- per plane in [xa, xe] the pass items form the y and z parts: a y item streams the TY + 14 nodes
  of column zc through a window of 8 and adds each face to the outputs it reaches; a z item does
  the same along its row segment of TY outputs, the last segment moved left to end at TZ;
- the march keeps the last 8 nodes and the 8 open outputs: each x face (face q-4 at plane q) goes
  to the open outputs q-7 .. q with tap 7-d, the newest output opens with its first face, and
  output q-7 is complete at plane q, when its plane's y+z part (formed 7 planes earlier) joins it.
Face weights are indexed from face -4 (w0 (nx+8, ny, nz) and so on); nodes outside the grid are
zero (the TMA fill), as are planes outside the chunk's march. No GPU is needed.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle.grid import staggered_coefficients

HALO = 7


def _node(phi, x, y, z):
    nx, ny, nz = phi.shape
    if 0 <= x < nx and 0 <= y < ny and 0 <= z < nz:
        return phi[x, y, z]
    return 0.0


def _weight(w, x, y, z):
    if 0 <= x < w.shape[0] and 0 <= y < w.shape[1] and 0 <= z < w.shape[2]:
        return w[x, y, z]
    return 0.0


def _pass_item(nodes, weights, tap, n_out):
    """A streamed pass item: len(nodes) = n_out + 14 nodes, n_out + 7 face weights -> n_out outputs."""
    acc = [0.0] * n_out
    win = [0.0] * 8
    for r, v in enumerate(nodes):
        win[r & 7] = v
        if r >= 7:
            rf = r - 7
            s = 0.0
            for j in range(8):
                s = tap[j] * win[(rf + j) & 7] + s
            f = weights[rf] * s
            for o in range(n_out):
                if rf - 7 <= o <= rf:
                    acc[o] = tap[7] * f if o == rf else tap[o + 7 - rf] * f + acc[o]
    return acc


def emulate_wide_apply(phi, faces, inv, pot, spacing, tz=36, xchunk=None, ty=8):
    TY = ty
    nx, ny, nz = phi.shape
    nzp = nz + (nz & 1)
    tap = [c / spacing for c in staggered_coefficients(8)]
    w0, w1, w2 = faces
    out = np.full(phi.shape, np.nan)
    xchunk = xchunk or nx
    for y0 in range(0, ny, TY):
        for z0 in range(0, nzp, tz):
            for xa in range(0, nx, xchunk):
                xe = min(xa + xchunk, nx) - 1
                q0 = xa - HALO if xa > 0 else 0
                yz = {}
                for q in range(xa, xe + 1):  # the pass groups' planes
                    part = np.zeros((TY, tz))
                    for zc in range(tz):  # y items: column z0+zc, outputs y0 .. y0+7
                        z = z0 + zc
                        if z >= nz:
                            continue
                        nodes = [_node(phi, q, y0 - HALO + r, z) for r in range(TY + 14)]
                        wts = [_weight(w1, q, y0 + rf, z) for rf in range(TY + 7)]  # faces y0-4+rf at y0+rf
                        part[:, zc] += _pass_item(nodes, wts, tap, TY)
                    for ry in range(TY):  # z items: row y0+ry, segments of TY outputs
                        y = y0 + ry
                        if y >= ny:
                            continue
                        for seg in range((tz + TY - 1) // TY):
                            zs = min(seg * TY, tz - TY)
                            first = seg * TY - zs
                            if z0 + zs >= nz:
                                continue
                            nodes = [_node(phi, q, y, z0 + zs - HALO + r) for r in range(TY + 14)]
                            wts = [_weight(w2, q, y, z0 + zs + rf) for rf in range(TY + 7)]
                            vals = _pass_item(nodes, wts, tap, TY)
                            for o in range(first, TY):
                                part[ry, zs + o] += vals[o]
                    yz[q] = part
                for ty in range(TY):  # the march: one thread per (y, z) column
                    y = y0 + ty
                    if y >= ny:
                        continue
                    for tzi in range(tz):
                        z = z0 + tzi
                        if z >= nz:
                            continue
                        phq = [0.0] * 8
                        acc = [0.0] * 8
                        for n in range(xe + HALO + 1 - q0):
                            q = q0 + n
                            g = n & 7
                            phq[g] = _node(phi, q, y, z)
                            s = 0.0
                            for j in range(8):
                                s = tap[j] * phq[(g + 1 + j) & 7] + s
                            face = _weight(w0, q, y, z) * s  # x face q-4, stored at index q
                            for d in range(1, 8):
                                acc[(g - d) & 7] = tap[7 - d] * face + acc[(g - d) & 7]
                            i = q - HALO
                            if i >= xa:
                                div = acc[(g + 1) & 7] + yz[i][ty, tzi]
                                out[i, y, z] = (0.5 * inv[i, y, z]) * div + phq[(g + 1) & 7] * pot[i, y, z]
                            acc[g] = tap[7] * face
    return out


@pytest.mark.parametrize("shape,ty,tz,xchunk", [((6, 9, 13), 8, 36, None), ((11, 10, 21), 8, 32, 5),
                                                ((9, 17, 40), 8, 36, 4), ((7, 27, 30), 13, 24, 4),
                                                ((5, 11, 9), 13, 24, None)])
def test_wide_kernel_emulation_is_the_apply(shape, ty, tz, xchunk):
    from types import SimpleNamespace

    from oracle.grid import Grid
    from oracle.operators import CuspHamiltonian

    rng = np.random.default_rng(sum(shape) + tz)
    nx, ny, nz = shape
    faces = (rng.uniform(0.5, 1.5, (nx + 8, ny, nz)), rng.uniform(0.5, 1.5, (nx, ny + 8, nz)),
             rng.uniform(0.5, 1.5, (nx, ny, nz + 8)))
    inv = rng.uniform(0.5, 1.5, shape)
    pot = rng.standard_normal(shape)
    spacing = 0.3
    grid = Grid(shape, spacing, (0.0, 0.0, 0.0))
    ham = CuspHamiltonian(grid, SimpleNamespace(face_weights=lambda order: faces), None,
                          bare=(pot.ravel(), inv.ravel(), rng.uniform(0.5, 1.5, shape).ravel()))
    phi = rng.standard_normal(shape)
    want = ham.apply(phi.ravel()).reshape(shape)
    got = emulate_wide_apply(phi, faces, inv, pot, spacing, tz=tz, xchunk=xchunk, ty=ty)
    assert not np.isnan(got).any(), "an output was never formed"
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-12 * np.abs(want).max())
