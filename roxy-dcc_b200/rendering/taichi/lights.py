"""Explicit light lists for next-event estimation.

Reference-compatible list: the emissive sphere slots in slot order
(rendering/taichi/extractor.py:36-50), picked uniformly.

Default list: emissive spheres plus every emissive triangle, picked in
proportion to emitted power (luminance x emission x area) through an alias
table (Vose, "A linear algorithm for generating random numbers with a given
distribution", IEEE TSE 1991).
"""
import numpy as np


def alias_table(weights):
    w = np.asarray(weights, dtype=np.float64)
    n = len(w)
    if n == 0:
        return np.zeros(0, np.float32), np.zeros(0, np.int32), np.zeros(0, np.float32)
    total = w.sum()
    if not np.isfinite(total) or total <= 0:
        w = np.ones(n)
        total = float(n)
    pdf = w / total
    scaled = pdf * n
    prob = np.ones(n, np.float64)
    alias = np.arange(n, dtype=np.int32)
    small = [i for i in range(n) if scaled[i] < 1.0]
    large = [i for i in range(n) if scaled[i] >= 1.0]
    while small and large:
        s = small.pop()
        g = large.pop()
        prob[s] = scaled[s]
        alias[s] = g
        scaled[g] = (scaled[g] + scaled[s]) - 1.0
        (small if scaled[g] < 1.0 else large).append(g)
    for i in large + small:
        prob[i] = 1.0
    return prob.astype(np.float32), alias, pdf.astype(np.float32)


def _lum(rgb):
    rgb = np.asarray(rgb, dtype=np.float64).reshape((-1, 3))
    return 0.2126 * rgb[:, 0] + 0.7152 * rgb[:, 1] + 0.0722 * rgb[:, 2]


def build_lights(slots, tri_v0, tri_v1, tri_v2, tri_mat, pal_type, pal_albedo, pal_emission, compat,
                 pal_texture=None, tri_index=None):
    """Light arrays for rx_scene_set_lights.

    slots: reference object-slot dicts; tri_*: triangles in caller order with
    palette index tri_mat; compat: sphere lights only, uniform pick;
    pal_texture: texture index per palette entry — textured emitters are
    left out (their radiance varies over the surface; BSDF rays find them);
    tri_index: scene triangle index of each tri_* row (None: row i is
    triangle i), reported as the triangle lights' sources.
    """
    kinds, p0, p1, p2, alb, em, area, src = [], [], [], [], [], [], [], []
    for si, s in enumerate(slots):
        if s["type"] == 0 and s["mat_type"] == 3 and s["emission"] > 0.0:
            kinds.append(0)
            src.append(si)
            p0.append(s["center"])
            p1.append([s["radius"], 0.0, 0.0])
            p2.append([0.0, 0.0, 0.0])
            alb.append(s["albedo"])
            em.append(s["emission"])
            area.append(np.pi * s["radius"] ** 2)
    n_sph = len(kinds)
    kind = np.array(kinds, np.int32)
    P0 = np.array(p0, np.float32).reshape((-1, 3))
    P1 = np.array(p1, np.float32).reshape((-1, 3))
    P2 = np.array(p2, np.float32).reshape((-1, 3))
    ALB = np.array(alb, np.float32).reshape((-1, 3))
    EM = np.array(em, np.float32)
    AREA = np.array(area, np.float32)
    SRC = np.array(src, np.int32)
    if not compat and tri_mat is not None and len(tri_mat):
        pt = np.asarray(pal_type)[tri_mat]
        pe = np.asarray(pal_emission)[tri_mat]
        keep = (pt == 3) & (pe > 0.0)
        if pal_texture is not None:
            keep &= np.asarray(pal_texture)[tri_mat] < 0
        sel = np.nonzero(keep)[0]
        if len(sel):
            a, b, c = tri_v0[sel], tri_v1[sel], tri_v2[sel]
            cr = np.cross((b - a).astype(np.float64), (c - a).astype(np.float64))
            tarea = 0.5 * np.linalg.norm(cr, axis=1)
            kind = np.concatenate([kind, np.ones(len(sel), np.int32)])
            P0 = np.concatenate([P0, a.astype(np.float32)])
            P1 = np.concatenate([P1, b.astype(np.float32)])
            P2 = np.concatenate([P2, c.astype(np.float32)])
            ALB = np.concatenate([ALB, np.asarray(pal_albedo, np.float32)[tri_mat[sel]]])
            EM = np.concatenate([EM, pe[sel].astype(np.float32)])
            AREA = np.concatenate([AREA, tarea.astype(np.float32)])
            SRC = np.concatenate([SRC, (sel if tri_index is None else np.asarray(tri_index)[sel]).astype(np.int32)])
    n = len(kind)
    if n == 0:
        return None
    if compat:
        prob, alias, pdf = np.ones(n, np.float32), np.arange(n, dtype=np.int32), np.full(n, 1.0 / n, np.float32)
    else:
        prob, alias, pdf = alias_table(_lum(ALB) * EM * AREA)
    return {"kind": kind, "p0": P0, "p1": P1, "p2": P2, "albedo": ALB, "emission": EM, "area": AREA,
            "pick_pdf": pdf, "alias_prob": prob, "alias_idx": alias, "n_spheres": n_sph,
            "source": SRC}  # object slot (sphere lights) or caller triangle index (triangle lights)
