"""numpy restatement of SparseDiffDMC.forward in training mode (weighted
average dual vertices, 4-triangle quad split).  TEST INFRASTRUCTURE ONLY.

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


def forward(voxel_coords, sdf, cube_idx, res, deform=None, beta=None, alpha=None, gamma=None, isovalue=0.0,
            weight_scale=0.99, dtype=np.float32):
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
