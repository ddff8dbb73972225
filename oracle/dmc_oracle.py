"""numpy restatement of SparseDiffDMC.forward: training mode (weighted
average dual vertices, 4-triangle quad split) and the QEF inference mode
(corner gradients, QEF dual vertices, 2-triangle split along the shorter
diagonal).  TEST INFRASTRUCTURE ONLY.

Follows atom3d/mesh_extractor/sparse_diffdmc.py:
  forward                 :76-232
  _normalize_weights      :234-253
  _compute_reg_loss       :255-261
  _compute_normals_from_gradient :263-287
  _identify_surf_cubes    :516-521
  _get_case_id_sparse     :524-579
  _identify_surf_edges    :582-599
  _compute_vd (weighted)  :601-780
  _triangulate (training) :782-826
  _linear_interp          :859-871
  QEF mode: _estimate_corner_gradients :451-513, crossing normals from
  corner gradients (_compute_vd) :610-650, _solve_qef_scatter :289-389,
  eval split (_triangulate) :798-805; the 3x3 systems are solved in FP64

dtype=np.float32 reproduces the reference's arithmetic order (pinned
against its golden outputs); dtype=np.float64 gives the FP64 function used
for central finite differences.
"""

from __future__ import annotations

import numpy as np

from atom3d_b200.mesh_extractor.dmc_tables import table

DMC = table("dmc_table")
NUM_VD = table("num_vd_table")
CHECK = table("check_table")
CUBE_CORNERS = np.array([[i & 1, (i >> 1) & 1, (i >> 2) & 1] for i in range(8)], np.int64)
CUBE_EDGES = np.array([0, 1, 1, 5, 4, 5, 0, 4, 2, 3, 3, 7, 6, 7, 2, 6, 2, 0, 3, 1, 7, 5, 6, 4], np.int64)


def linear_interp(w, x):
    """w [..., 2, 1 or C], x [..., 2, C]: (x0*w1 - x1*w0) / (w1 - w0)."""
    ew = np.concatenate([w[..., 1:2, :], -w[..., 0:1, :]], axis=-2)
    den = ew[..., 0, :] + ew[..., 1, :]
    num = x[..., 0, :] * ew[..., 0, :] + x[..., 1, :] * ew[..., 1, :]
    return num / den


def qef_solve(n, r, eg_vd, cen, c_ctr, V, lam):
    """The least-squares system _solve_qef_scatter (:316-367) assembles.

    Its slot scatter (group_offsets.scatter_ with repeated indices keeps the
    last position on the CPU) gives the j-th of a vertex's k constraints the
    row (j - (k - 1)) mod 10: the last one row 0, the others rows 9, 8, 7,
    6, 5, 4.  The regularisation then sets element (7, 0), (8, 1), (9, 2) to
    sqrt(lambda) -- keeping the other two components of a constraint placed
    there -- and rows 7-9 of b to sqrt(lambda) (centre - centroid).  This
    restates that system (it reproduces the reference's CPU outputs); it is
    solved through its 3x3 normal equations in FP64.
    """
    K = n.shape[0]
    last = np.zeros(V, np.int64)
    last[eg_vd] = np.arange(K)
    row = (np.arange(K) - last[eg_vd]) % 10
    A = np.zeros((V, 10, 3))
    b = np.zeros((V, 10))
    A[eg_vd, row] = n
    b[eg_vd, row] = r
    sl = np.sqrt(lam)
    A[:, 7, 0] = sl
    A[:, 8, 1] = sl
    A[:, 9, 2] = sl
    b[:, 7:10] = (c_ctr - cen) * sl
    ata = np.einsum("vri,vrj->vij", A, A)
    atb = np.einsum("vri,vr->vi", A, b)
    return np.linalg.solve(ata, atb[..., None])[..., 0]


def corner_gradients(x, sf, ci, dtype=np.float32):
    """Least-squares SDF gradient at every corner from all incident cube
    edges (_estimate_corner_gradients)."""
    f = dtype
    M = x.shape[0]
    ue = np.unique(ci[:, CUBE_EDGES].reshape(-1, 2), axis=0)
    i0, i1 = ue[:, 0], ue[:, 1]
    ev = x[i1] - x[i0]
    el = np.maximum(np.sqrt((ev * ev).sum(-1, keepdims=True)), f(1e-8))
    ed = ev / el
    gp = (sf[i1] - sf[i0]) / el[:, 0]
    outer = ed[:, :, None] * ed[:, None, :]
    fwd = gp[:, None] * ed
    dtd = np.zeros((M, 3, 3), np.float64)
    dtb = np.zeros((M, 3), np.float64)
    np.add.at(dtd, i0, outer)
    np.add.at(dtd, i1, outer)
    np.add.at(dtb, i0, fwd)
    np.add.at(dtb, i1, -fwd)
    dtd += 1e-4 * np.eye(3)[None]
    g = np.linalg.solve(dtd, dtb[..., None])[..., 0]
    g[np.isnan(g).any(-1)] = 0.0
    return g.astype(f)


def forward(voxel_coords, sdf, cube_idx, res, deform=None, beta=None, alpha=None, gamma=None, isovalue=0.0,
            weight_scale=0.99, dtype=np.float32, mode="weighted_avg", qef_reg_scale=1e-2, corner_grads=None):
    f = dtype
    vox = np.asarray(voxel_coords, np.int64)
    ci = np.asarray(cube_idx, np.int64)
    s = np.asarray(sdf).astype(f)
    M = s.shape[0]
    # 1-2: corner positions
    pos = np.zeros((M, 3), f)
    cpos = (vox[:, None, :] + CUBE_CORNERS[None]).reshape(-1, 3).astype(f)
    pos[ci.reshape(-1)] = cpos
    ws = f(2.0 / res)
    x = pos * ws - f(1.0)
    if deform is not None:
        x = x + np.asarray(deform).astype(f)
    sf = s - f(isovalue)
    # 4: surface cubes
    occ = sf < 0
    occ8 = occ[ci.reshape(-1)].reshape(-1, 8)
    osum = occ8.sum(-1)
    surf = (osum > 0) & (osum < 8)
    empty = dict(vertices=np.zeros((0, 3), f), faces=np.zeros((0, 3), np.int64), L_dev=np.zeros(0, f),
                 p_alpha=np.zeros((0, 3), f), n_alpha=np.zeros((0, 3), f))
    if surf.sum() == 0:
        return empty
    N = vox.shape[0]
    # 5: weights
    beta_o = (np.tanh(np.asarray(beta).astype(f)) * f(weight_scale) + f(1)) if beta is not None else np.ones((N, 12), f)
    alpha_o = (np.tanh(np.asarray(alpha).astype(f)) * f(weight_scale) + f(1)) if alpha is not None else np.ones((N, 8), f)
    beta_s, alpha_s = beta_o[surf], alpha_o[surf]
    # 6: case ids with the C16/C19 fix
    case = (occ8[surf].astype(np.int64) * (1 << np.arange(8))).sum(-1)
    prob = CHECK[case]
    to_check = prob[:, 0] == 1
    if to_check.any():
        pc = vox[surf][to_check]
        sub = prob[to_check]
        adj = pc + sub[:, 1:4]
        within = (adj >= 0).all(-1) & (adj < res).all(-1)
        if within.any():
            ph = pc[:, 0] * (res * res) + pc[:, 1] * res + pc[:, 2]
            sh = np.sort(ph)
            ah = adj[within, 0] * (res * res) + adj[within, 1] * res + adj[within, 2]
            p = np.clip(np.searchsorted(sh, ah), 0, sh.shape[0] - 1)
            found = sh[p] == ah
            if found.any():
                idx = np.arange(case.shape[0])[to_check][within][found]
                case = case.copy()
                case[idx] = sub[within][found][:, -1]
    # 7: surface edges
    ci_s = ci[surf]
    all_e = ci_s[:, CUBE_EDGES].reshape(-1, 2)
    ue, inv, cnt = np.unique(all_e, axis=0, return_inverse=True, return_counts=True)
    inv = inv.reshape(-1)
    mask_e = occ[ue.reshape(-1)].reshape(-1, 2).sum(-1) == 1
    surf_edges_mask = mask_e[inv]
    counts = cnt[inv]
    mapping = -np.ones(ue.shape[0], np.int64)
    mapping[mask_e] = np.arange(mask_e.sum())
    idx_map = mapping[inv]
    surf_edges = ue[mask_e]
    # 8: dual vertices
    sx = x[surf_edges.reshape(-1)].reshape(-1, 2, 3)
    ss = sf[surf_edges.reshape(-1)].reshape(-1, 2, 1)
    zc = linear_interp(ss, sx)
    p0, p1 = sx[:, 0], sx[:, 1]
    ev = p1 - p0
    el = np.sqrt((ev * ev).sum(-1, keepdims=True)) + f(1e-8)
    ed = ev / el
    gm = (ss[:, 1] - ss[:, 0]) / el
    nrm = ed * np.sign(gm)
    nl = np.sqrt((nrm * nrm).sum(-1, keepdims=True))
    normals = nrm / np.maximum(nl, f(1e-12))
    idx_map12 = idx_map.reshape(-1, 12)
    num_vd = NUM_VD[case]
    eg, eg_vd, eg_cube, vd_ne = [], [], [], []
    total = 0
    for num in np.unique(num_vd):
        if num == 0:
            continue
        cur = np.nonzero(num_vd == num)[0]
        tab = DMC[case[cur], :num].reshape(-1, num * 7)
        gvd = (np.arange(cur.shape[0] * num)[:, None].repeat(7, 1) + total).reshape(tab.shape)
        gcube = np.repeat(cur[:, None], num * 7, 1)
        m = tab != -1
        eg.append(tab[m])
        eg_vd.append(gvd[m])
        eg_cube.append(gcube[m])
        vd_ne.append(m.reshape(-1, 7).sum(-1))
        total += cur.shape[0] * num
    eg = np.concatenate(eg)
    eg_vd = np.concatenate(eg_vd)
    eg_cube = np.concatenate(eg_cube)
    vd_ne = np.concatenate(vd_ne)
    flat = eg_cube * 12 + eg
    ig = idx_map12.reshape(-1)[flat]
    zg = zc[ig]
    sg = ss[ig]
    xg = sx[ig]
    ng = normals[ig]
    a_pairs = alpha_s[:, CUBE_EDGES].reshape(-1, 12, 2)
    ag = a_pairs.reshape(-1, 2)[flat][..., None]
    ueg = linear_interp(sg * ag, xg)
    bg = beta_s.reshape(-1)[flat][:, None]
    V = total
    if mode == "qef":
        G = corner_grads if corner_grads is not None else corner_gradients(x, sf, ci, f)
        s0e, s1e = ss[:, 0, 0], ss[:, 1, 0]
        t = np.clip(s0e / (s0e - s1e + f(1e-8)), 0, 1)[:, None]
        g0, g1 = G[surf_edges[:, 0]], G[surf_edges[:, 1]]
        w0 = np.sqrt((g0 * g0).sum(-1, keepdims=True)) * (1 - t)
        w1 = np.sqrt((g1 * g1).sum(-1, keepdims=True)) * t
        den = w0 + w1
        gc = (w0 * g0 + w1 * g1) / np.maximum(den, f(1e-8))
        gc = np.where(den > f(1e-6), gc, normals)
        all_n = gc / np.maximum(np.sqrt((gc * gc).sum(-1, keepdims=True)), f(1e-12))
        ng = all_n[ig]
        cnt_v = np.zeros(V, np.float64)
        np.add.at(cnt_v, eg_vd, 1.0)
        cen = np.zeros((V, 3), np.float64)
        np.add.at(cen, eg_vd, zg.astype(np.float64))
        cen = cen / np.maximum(cnt_v, 1)[:, None]
        vd_cube = np.zeros(V, np.int64)
        vd_cube[eg_vd] = eg_cube
        cv = x[ci_s[vd_cube]].astype(np.float64)
        c_ctr, c_min, c_max = cv.mean(1), cv.min(1), cv.max(1)
        n64 = ng.astype(np.float64)
        r = (n64 * (zg.astype(np.float64) - cen[eg_vd])).sum(-1)
        delta = qef_solve(n64, r, eg_vd, cen, c_ctr, V, float(qef_reg_scale))
        vd = delta + cen
        bad = np.isnan(vd).any(-1)
        margin = c_max - c_min
        bad |= (vd < c_min - margin).any(-1) | (vd > c_max + margin).any(-1)
        vd[bad] = cen[bad]
        vd = vd.astype(f)
    else:
        bsum = np.zeros((V, 1), f)
        np.add.at(bsum, eg_vd, bg)
        acc = np.zeros((V, 3), f)
        np.add.at(acc, eg_vd, ueg * bg)
        vd = acc / (bsum + f(1e-8))
    dist = np.sqrt(((zg - vd[eg_vd]) ** 2).sum(-1))
    mean = np.zeros(V, f)
    np.add.at(mean, eg_vd, dist)
    mean = mean / vd_ne.astype(f)
    ldev = np.abs(dist - mean[eg_vd])
    vd_idx_map = np.zeros(case.shape[0] * 12, np.int64)
    vd_idx_map[flat] = eg_vd
    # 9: triangulate (training split)
    gmask = (counts == 4) & surf_edges_mask
    group = idx_map.reshape(-1)[gmask]
    vdi = vd_idx_map[gmask]
    order = np.argsort(group, kind="stable")
    eidx = group[order]
    quad = vdi[order].reshape(-1, 4)
    se = sf[surf_edges[eidx.reshape(-1, 4)[:, 0]].reshape(-1)].reshape(-1, 2)
    flip = se[:, 0] > 0
    q = quad.copy()
    q[flip] = quad[flip][:, [0, 1, 3, 2]]
    q[~flip] = quad[~flip][:, [2, 3, 1, 0]]
    vq = vd[q.reshape(-1)].reshape(-1, 4, 3)
    if mode == "qef":
        d02 = vq[:, 0] - vq[:, 2]
        d13 = vq[:, 1] - vq[:, 3]
        m = np.sqrt((d02 * d02).sum(-1)) < np.sqrt((d13 * d13).sum(-1))
        faces = np.where(m[:, None], q[:, [0, 1, 2, 0, 2, 3]], q[:, [0, 1, 3, 3, 1, 2]]).reshape(-1, 3)
        return dict(vertices=vd, faces=faces, L_dev=ldev, p_alpha=ueg, n_alpha=ng)
    centre = vq.mean(axis=1).astype(f)
    cidx = np.arange(centre.shape[0]) + V
    verts = np.concatenate([vd, centre], 0)
    fc = q[:, [0, 1, 1, 2, 2, 3, 3, 0]].reshape(-1, 4, 2)
    faces = np.concatenate([fc, np.repeat(cidx[:, None, None], 4, 1)], -1).reshape(-1, 3)
    return dict(vertices=verts, faces=faces, L_dev=ldev, p_alpha=ueg, n_alpha=ng)


def loss_vertices_sq(*args, **kw):
    """Sum of squared vertex norms (the benchmark/test loss)."""
    out = forward(*args, **kw)
    return float((out["vertices"].astype(np.float64) ** 2).sum())
