"""The oracle's gcbc_go (or_gcbc_go: every face code, single rank) pinned by
what the characteristic closures must do, checked on the CPU:
  * non-reflective faces: the same correction as the fused x-face closure
    or_gcbc_x;
  * with sbcc = 1/J on the face plane, the characteristic form of the updated
    J de at a face point is the closure's target: incoming acoustic waves
    zeroed (non-reflective), the incoming wave reflected from the outgoing
    one with the frame acceleration and the relaxed normal velocity (walls),
    the incoming waves taken from the neighbour (curvilinear interface)."""
import numpy as np

import oracle as O

GAM = 1.4


def case(dims, seed):
    r = np.random.default_rng(seed)
    n = int(np.prod(dims))
    q = O.tgv_init(dims, 0.3, 1e-3, seed)
    q[3 * n:4 * n] = 0.05 * q[:n] * np.sin(np.arange(n) * 0.01)
    _, p = O.thermo(q)
    de = 0.1 * r.standard_normal(5 * n)
    yaco = 1.0 + 0.2 * r.random(n)
    F = (dims[1] * dims[2], dims[0] * dims[2], dims[0] * dims[1])
    drva, cm = [], []
    for a in range(3):
        drva.append(r.standard_normal(10 * F[a]))
        c = np.zeros((2, 3, F[a]))
        c[:, a, :] = 1.0
        c += 0.2 * r.standard_normal((2, 3, F[a]))
        c /= np.linalg.norm(c, axis=1, keepdims=True)
        cm.append(c.ravel().copy())
    return q, p, de, yaco, drva, cm, F


def face_points(dims, a, ip):
    """Linear indices of the face points of face ip of axis a, in face order."""
    lxi, let, lze = dims
    idx = np.arange(lxi * let * lze).reshape(lze, let, lxi)
    if a == 0:
        return idx[:, :, -1 if ip else 0].ravel()
    if a == 1:
        return idx[:, -1 if ip else 0, :].ravel()
    return idx[-1 if ip else 0, :, :].ravel()


def plane_weights(dims, yaco, faces):
    sbcc = np.zeros(int(np.prod(dims)))
    for a, ip in faces:
        pts = face_points(dims, a, ip)
        sbcc[pts] = 1.0 / yaco[pts]
    return sbcc


def characteristic(q, p, de, yaco, cm, dims, a, ip):
    """xtq2r (J de) at the face points of face (a, ip), through the oracle's
    setup step (a wall code: characteristic of the full right-hand side)."""
    F = cm[a].size // 6
    nbc = [[45] * 3, [45] * 3]
    nbc[ip][a] = 20
    drva = [np.zeros(10 * (cm[b].size // 6)) for b in range(3)]
    de_c = de.copy()
    O.gcbc_go(drva, cm, [None] * 3, q, de_c, p, yaco, np.zeros_like(yaco), (0, 0, 0), (0, 0, 0), dims, 0.0, nbc)
    return drva[a].reshape(2, 5, F)[ip]


def point_state(q, p, cm, dims, a, ip, umf):
    n = int(np.prod(dims))
    pts = face_points(dims, a, ip)
    F = pts.size
    c = cm[a].reshape(2, 3, F)[ip]
    rho = q[pts]
    ve = np.stack([q[(1 + k) * n + pts] / rho for k in range(3)])
    ao = np.sqrt(GAM * p[pts] / rho)
    vn = (c * ve).sum(0)
    vs = (c * np.asarray(umf)[:, None]).sum(0)
    return rho, ao, vn, vs, c


def test_non_reflective_equals_fused_x_closure():
    dims = (20, 16, 12)
    q, p, de, yaco, drva, cm, F = case(dims, 1)
    m = O.uniform_metrics(*dims)
    yc = np.full(int(np.prod(dims)), m.c_yaco)
    sbcc = np.random.default_rng(2).random(yc.size)
    nbc = [[10, 45, 45], [10, 45, 45]]
    de1 = de.copy()
    O.gcbc_x(de1, drva[0].copy(), cm[0], q, sbcc, m, dims, nbc)
    de2 = de.copy()
    O.gcbc_go([drva[0].copy(), None, None], cm, [None] * 3, q, de2, p, yc, sbcc, (0, 0, 0), (0, 0, 0), dims,
              0.0, nbc)
    c1, c2 = de1 - de, de2 - de
    assert np.abs(c1).max() > 0
    assert np.abs(c1 - c2).max() / np.abs(c1).max() < 1e-13


def test_closures_reach_their_characteristic_targets():
    """One axis at a time (both faces coded, the other axes periodic; sbcc =
    1/J on the two face planes only), every face code on every axis."""
    dims = (20, 16, 12)
    q, p, de, yaco, drva, cm, F = case(dims, 3)
    umf, dudtmf, dtwi = (0.02, -0.01, 0.015), (0.3, -0.2, 0.1), 25.0
    for codes in ((10, 25), (20, 10), (30, 30)):
        for a in range(3):
            nbc = [[45] * 3, [45] * 3]
            nbc[0][a], nbc[1][a] = codes
            sbcc = plane_weights(dims, yaco, [(a, 0), (a, 1)])
            drva_c = [x.copy() for x in drva]
            drvb = [np.zeros(10 * f) for f in F]
            de_new = de.copy()
            O.gcbc_go(drva_c, cm, drvb, q, de_new, p, yaco, sbcc, umf, dudtmf, dims, dtwi, nbc)
            for ip in range(2):
                code = nbc[ip][a]
                ra0 = 1.0 - 2.0 * ip
                rho, ao, vn, vs, c = point_state(q, p, cm, dims, a, ip, umf)
                cha = drva_c[a].reshape(2, 5, F[a])[ip]          # the closure's characteristic input
                old = characteristic(q, p, de, yaco, cm, dims, a, ip)
                after = characteristic(q, p, de_new, yaco, cm, dims, a, ip)
                scale = np.abs(old).max() + np.abs(cha).max()
                if code == 10:
                    target = old.copy()
                    s3, s4 = ra0 * (vn + vs + ao) > 0, ra0 * (vn + vs - ao) > 0
                    target[3, s3] -= cha[3, s3]
                    target[4, s4] -= cha[4, s4]
                    assert np.abs(after - target).max() < 1e-12 * scale, (a, ip, code)
                elif code in (20, 25):
                    assert np.abs(cha - old).max() < 1e-13 * scale       # walls start from J de
                    acc = (c * np.asarray(dudtmf)[:, None]).sum(0)
                    w = 2.0 * ra0 * rho / ao * (acc + dtwi * (vn + vs))
                    assert np.abs(after[3 + ip] - (after[4 - ip] + w)).max() < 1e-12 * scale, (a, ip, code)
                    keep = [v for v in range(5) if v != 3 + ip]
                    assert np.abs(after[keep] - old[keep]).max() < 1e-12 * scale, (a, ip, code)
                else:
                    nb = drvb[a].reshape(2, 5, F[a])[ip]
                    assert np.array_equal(nb, drva_c[a].reshape(2, 5, F[a])[1 - ip])  # GCIC self exchange
                    target = old.copy()
                    sel = ra0 * (vn + vs) > 0
                    target[:3, sel] = nb[:3, sel]
                    s3, s4 = ra0 * (vn + vs + ao) > 0, ra0 * (vn + vs - ao) > 0
                    target[3, s3] = nb[3, s3]
                    target[4, s4] = nb[4, s4]
                    assert np.abs(after - target).max() < 1e-12 * scale, (a, ip, code)
