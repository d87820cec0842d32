"""CPU emulation of the deterministic scatter (E^T) used by pa_apply_kernel,
merge_and_store and fixup_kernel, fed with oracle element matrices.

The emulation follows the kernel's rules step by step: x merge (lane l gets
lane l-1's a=P face), y merge (warp w gets warp w-1's b=P row), z carry,
owned stores / face slots with x > y > z priority, and the fix-up sum over
neighbour items in (dz, dy, dx) order.  It must reproduce the oracle apply,
for tile counts > 1 in every direction and ragged last tiles.
"""
import numpy as np
import pytest

from conftest import oracle as O


def emulate(mesh, coef, x, WY, TZ, ess_bits=0):
    p, D = mesh.p, mesh.p + 1
    nx, ny, nz = mesh.nx, mesh.ny, mesh.nz
    NK, NJ, NI = mesh.shape
    ntx, nty, ntz = -(-nx // 32), -(-ny // WY), -(-nz // TZ)
    SX, SY, SZ = 32 * p, WY * p, TZ * p
    fxs, fys, fzs = (SZ + 1) * (SY + 1), (SZ + 1) * (SX + 1), (SY + 1) * (SX + 1)
    fstride = fxs + fys + fzs
    face = np.full(ntx * nty * ntz * fstride, np.nan)
    y = np.full(mesh.ndofs, np.nan)
    X = x.reshape(NK, NJ, NI)
    mask = O.ess_mask(mesh, ess_bits).reshape(NK, NJ, NI)
    Ke = {}

    def elem_out(ex, ey, ez):
        e = (ez * ny + ey) * nx + ex
        if e not in Ke:
            Ke[e] = O.element_matrix(mesh, e, coef)
        u = X[ez * p:ez * p + D, ey * p:ey * p + D, ex * p:ex * p + D].copy()
        u[mask[ez * p:ez * p + D, ey * p:ey * p + D, ex * p:ex * p + D] == 1] = 0.0
        return (Ke[e] @ u.ravel()).reshape(D, D, D)  # [c][b][a]

    for item in range(ntx * nty * ntz):
        tx, ty, tz = item % ntx, (item // ntx) % nty, item // (ntx * nty)
        nl = min(TZ, nz - tz * TZ)
        lane_last = min(31, nx - 1 - tx * 32)
        w_last = min(WY - 1, ny - 1 - ty * WY)
        I0, J0, K0 = tx * SX, ty * SY, tz * SZ
        carry = np.zeros((WY, 32, D, D))
        for lz in range(nl):
            ez = tz * TZ + lz
            out = np.zeros((WY, 32, D, D, D))
            for w in range(WY):
                for l in range(32):
                    ex, ey = tx * 32 + l, ty * WY + w
                    if ex < nx and ey < ny:
                        out[w, l] = elem_out(ex, ey, ez)
            # x merge
            for w in range(WY):
                sh = out[w, :, :, :, p].copy()
                out[w, 1:, :, :, 0] += sh[:-1]
            # y merge (reads the pre-merge b=P row of warp w-1 after its x merge)
            rows = out[:, :, :, p, :].copy()
            out[1:, :, :, 0, :] += rows[:-1]
            # z carry
            if lz > 0:
                out[:, :, 0, :, :] += carry
            carry = out[:, :, p, :, :].copy()
            last = lz == nl - 1
            for w in range(WY):
                for l in range(32):
                    ex, ey = tx * 32 + l, ty * WY + w
                    if not (ex < nx and ey < ny):
                        continue
                    for c in range(D):
                        if c == p and not last:
                            continue
                        K = K0 + p * lz + c
                        zhi = c == p and ez != nz - 1
                        for b in range(D):
                            if b == p and w != w_last:
                                continue
                            J = J0 + p * w + b
                            yhi = b == p and ey != ny - 1
                            for a in range(D):
                                if a == p and l != lane_last:
                                    continue
                                I = I0 + p * l + a
                                xhi = a == p and ex != nx - 1
                                v = out[w, l, c, b, a]
                                base = item * fstride
                                if xhi:
                                    face[base + (K - K0) * (SY + 1) + (J - J0)] = v
                                elif yhi:
                                    face[base + fxs + (K - K0) * (SX + 1) + (I - I0)] = v
                                elif zhi:
                                    face[base + fxs + fys + (J - J0) * (SX + 1) + (I - I0)] = v
                                else:
                                    if mask[K, J, I]:
                                        v = X[K, J, I]
                                    y[(K * NJ + J) * NI + I] = v
    # fix-up
    for K in range(NK):
        for J in range(NJ):
            for I in range(NI):
                sx = int(0 < I < NI - 1 and I % SX == 0)
                sy = int(0 < J < NJ - 1 and J % SY == 0)
                sz = int(0 < K < NK - 1 and K % SZ == 0)
                if not (sx or sy or sz) or mask[K, J, I]:
                    continue
                tx, ty, tz = min(I // SX, ntx - 1), min(J // SY, nty - 1), min(K // SZ, ntz - 1)
                d = (K * NJ + J) * NI + I
                s = y[d]
                for dz in range(sz + 1):
                    for dy in range(sy + 1):
                        for dx in range(sx + 1):
                            if not (dx or dy or dz):
                                continue
                            nb = ((tz - dz) * nty + (ty - dy)) * ntx + (tx - dx)
                            I0, J0, K0 = (tx - dx) * SX, (ty - dy) * SY, (tz - dz) * SZ
                            base = nb * fstride
                            if dx:
                                s += face[base + (K - K0) * (SY + 1) + (J - J0)]
                            elif dy:
                                s += face[base + fxs + (K - K0) * (SX + 1) + (I - I0)]
                            else:
                                s += face[base + fxs + fys + (J - J0) * (SX + 1) + (I - I0)]
                y[d] = s
    return y


@pytest.mark.parametrize("shape,p,WY,TZ,ess", [
    ((33, 5, 5), 1, 4, 2, 0),
    ((34, 9, 7), 2, 4, 3, 63),
    ((35, 3, 4), 3, 2, 2, 16 | 2),
    ((3, 2, 2), 2, 4, 8, 0),
])
def test_scatter_emulation_matches_oracle(shape, p, WY, TZ, ess):
    mesh = O.Mesh(*shape, p)
    rng = np.random.default_rng(sum(shape))
    coef = O.Coef(O.DIFF, kappa_q=np.exp(rng.normal(size=mesh.n_elem * (p + 1) ** 3)))
    x = rng.normal(size=mesh.ndofs)
    y = emulate(mesh, coef, x, WY, TZ, ess)
    assert not np.isnan(y).any(), "a DOF was never written"
    ref = O.apply_constrained(mesh, coef, O.ess_mask(mesh, ess), x) if ess else O.pa_apply(mesh, coef, x)
    assert np.linalg.norm(y - ref) <= 1e-12 * np.linalg.norm(ref)


def fixup_rows_visit(NI, NJ, NK, p, WY, TZ, ntx, nty, ntz, ess):
    """The DOFs fixup_row_t visits, row by row, with the owner item and plane
    flags it passes to fixup_acc: (I, J, K) -> (tx, ty, tz, sx, sy, sz)."""
    SX, SY, SZ = 32 * p, WY * p, TZ * p
    rx, ry, rz = (ntx - 1) * NK, (nty - 1) * NK, (ntz - 1) * NJ
    ess_i = lambda I: (ess & 16 and I == 0) or (ess & 32 and I == NI - 1)  # noqa: E731
    ess_j = lambda J: (ess & 4 and J == 0) or (ess & 8 and J == NJ - 1)  # noqa: E731
    ess_k = lambda K: (ess & 1 and K == 0) or (ess & 2 and K == NK - 1)  # noqa: E731
    on_x = lambda I: 0 < I < NI - 1 and I % SX == 0  # noqa: E731
    seen = {}
    for r in range(rx + ry + rz):
        if r < rx:
            pl, K = divmod(r, NK)
            I, tx = (pl + 1) * SX, pl + 1
            if ess_k(K):
                continue
            sz, tz = int(0 < K < NK - 1 and K % SZ == 0), min(K // SZ, ntz - 1)
            for J in range(NJ):
                if ess_j(J):
                    continue
                sy, ty = int(0 < J < NJ - 1 and J % SY == 0), min(J // SY, nty - 1)
                assert (I, J, K) not in seen
                seen[(I, J, K)] = (tx, ty, tz, 1, sy, sz)
        elif r < rx + ry:
            pl, K = divmod(r - rx, NK)
            J, ty = (pl + 1) * SY, pl + 1
            if ess_k(K):
                continue
            sz, tz = int(0 < K < NK - 1 and K % SZ == 0), min(K // SZ, ntz - 1)
            for I in range(NI):
                if on_x(I) or ess_i(I):
                    continue
                assert (I, J, K) not in seen
                seen[(I, J, K)] = (min(I // SX, ntx - 1), ty, tz, 0, 1, sz)
        else:
            pl, J = divmod(r - rx - ry, NJ)
            K, tz = (pl + 1) * SZ, pl + 1
            if (0 < J < NJ - 1 and J % SY == 0) or ess_j(J):
                continue
            ty = min(J // SY, nty - 1)
            for I in range(NI):
                if on_x(I) or ess_i(I):
                    continue
                assert (I, J, K) not in seen
                seen[(I, J, K)] = (min(I // SX, ntx - 1), ty, tz, 0, 0, 1)
    return seen


@pytest.mark.parametrize("shape,p,WY,TZ,ess", [
    ((33, 5, 5), 1, 4, 2, 0),
    ((70, 9, 7), 2, 4, 3, 63),
    ((65, 7, 9), 3, 2, 2, 16 | 2 | 8),
    ((3, 2, 2), 2, 4, 8, 0),
    ((64, 8, 16), 2, 4, 8, 32 | 1 | 4),
])
def test_fixup_rows_cover_each_shared_dof_once(shape, p, WY, TZ, ess):
    """The row decomposition of the fix-up kernel visits exactly the shared,
    non-essential DOFs, once each, with the owner item and plane flags of the
    per-DOF rule (the plane flags and owner item fixup_acc is given)."""
    nx, ny, nz = shape
    NI, NJ, NK = nx * p + 1, ny * p + 1, nz * p + 1
    ntx, nty, ntz = -(-nx // 32), -(-ny // WY), -(-nz // TZ)
    SX, SY, SZ = 32 * p, WY * p, TZ * p
    seen = fixup_rows_visit(NI, NJ, NK, p, WY, TZ, ntx, nty, ntz, ess)
    assert seen == per_dof_rule(NI, NJ, NK, SX, SY, SZ, ntx, nty, ntz, ess)


def per_dof_rule(NI, NJ, NK, SX, SY, SZ, ntx, nty, ntz, ess):
    """The per-DOF classification of the fix-up: shared (on a plane between
    items) and not essential -> owner item and plane flags."""
    want = {}
    for K in range(NK):
        for J in range(NJ):
            for I in range(NI):
                sx = int(0 < I < NI - 1 and I % SX == 0)
                sy = int(0 < J < NJ - 1 and J % SY == 0)
                sz = int(0 < K < NK - 1 and K % SZ == 0)
                e = ((ess & 1 and K == 0) or (ess & 2 and K == NK - 1) or (ess & 4 and J == 0) or
                     (ess & 8 and J == NJ - 1) or (ess & 16 and I == 0) or (ess & 32 and I == NI - 1))
                if (sx or sy or sz) and not e:
                    want[(I, J, K)] = (min(I // SX, ntx - 1), min(J // SY, nty - 1), min(K // SZ, ntz - 1),
                                       sx, sy, sz)
    return want


def fixup_owner_visit(NI, NJ, NK, p, WY, TZ, ntx, nty, ntz, ess):
    """The DOFs the fused fix-up (fixup_owner, run once per item by the last of
    its contributors to arrive) visits, with the flags it passes to fixup_acc."""
    SX, SY, SZ = 32 * p, WY * p, TZ * p
    seen = {}
    for oz in range(ntz):
        for oy in range(nty):
            for ox in range(ntx):
                if (1 + (ox > 0)) * (1 + (oy > 0)) * (1 + (oz > 0)) == 1:
                    continue
                I0, J0, K0 = ox * SX, oy * SY, oz * SZ
                I1 = NI - 1 if ox == ntx - 1 else I0 + SX - 1
                J1 = NJ - 1 if oy == nty - 1 else J0 + SY - 1
                K1 = NK - 1 if oz == ntz - 1 else K0 + SZ - 1
                ia, ja = I0 + (ox > 0), J0 + (oy > 0)
                nI, nJ, nJy, nK = I1 - ia + 1, J1 - J0 + 1, J1 - ja + 1, K1 - K0 + 1
                cx = nJ * nK if ox > 0 else 0
                cy = nI * nK if oy > 0 else 0
                cz = nI * nJy if oz > 0 else 0
                for t in range(cx + cy + cz):
                    if t < cx:
                        k, j = divmod(t, nJ)
                        I, J, K = I0, J0 + j, K0 + k
                        f = (1, int(J == J0 and oy > 0), int(K == K0 and oz > 0))
                    elif t < cx + cy:
                        k, i = divmod(t - cx, nI)
                        I, J, K = ia + i, J0, K0 + k
                        f = (0, 1, int(K == K0 and oz > 0))
                    else:
                        j, i = divmod(t - cx - cy, nI)
                        I, J, K = ia + i, ja + j, K0
                        f = (0, 0, 1)
                    e = ((ess & 1 and K == 0) or (ess & 2 and K == NK - 1) or (ess & 4 and J == 0) or
                         (ess & 8 and J == NJ - 1) or (ess & 16 and I == 0) or (ess & 32 and I == NI - 1))
                    if e:
                        continue
                    assert 0 <= I < NI and 0 <= J < NJ and 0 <= K < NK
                    assert (I, J, K) not in seen
                    seen[(I, J, K)] = (ox, oy, oz) + f
    return seen


@pytest.mark.parametrize("shape,p,WY,TZ,ess", [
    ((33, 5, 5), 1, 4, 2, 0),
    ((70, 9, 7), 2, 4, 3, 63),
    ((65, 7, 9), 3, 2, 2, 16 | 2 | 8),
    ((3, 2, 2), 2, 4, 8, 0),
    ((64, 8, 16), 2, 4, 8, 32 | 1 | 4),
    ((4, 4, 4), 1, 4, 1, 63),
    ((96, 12, 8), 1, 4, 4, 63),
])
def test_fused_fixup_owners_match_rows(shape, p, WY, TZ, ess):
    """The per-owner enumeration of the fused fix-up and the row decomposition
    of fixup_kernel visit the same DOFs with the same owner and plane flags."""
    nx, ny, nz = shape
    NI, NJ, NK = nx * p + 1, ny * p + 1, nz * p + 1
    ntx, nty, ntz = -(-nx // 32), -(-ny // WY), -(-nz // TZ)
    rows = fixup_rows_visit(NI, NJ, NK, p, WY, TZ, ntx, nty, ntz, ess)
    owners = fixup_owner_visit(NI, NJ, NK, p, WY, TZ, ntx, nty, ntz, ess)
    assert owners == rows == per_dof_rule(NI, NJ, NK, 32 * p, WY * p, TZ * p, ntx, nty, ntz, ess)
