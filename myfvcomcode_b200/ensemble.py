"""Batched ensembles: members stepped together.

Members that share a mesh and layer count are stepped as one *union* model: the disjoint
union of the member meshes, every index array offset by its member's node, cell, edge,
half-edge, open-boundary and river offsets (index 0, FVCOM's ghost, stays 0).  Each
member's gather lists stay inside the member and keep their order, so a member of a
union run is bitwise equal to the same member run alone in FP64.  Models of different
meshes or layer counts are stepped together by ``fvg_group_*`` (one CUDA graph holding
one internal step of each model on its own branch).

Perturbations of a member (EnKF-style, seeded): wind speed scaled by a factor uniform in
[1-w, 1+w], open-boundary tidal amplitudes by a factor uniform in [1-a, 1+a], and the
initial temperature shifted by an offset drawn from N(0, sigma_T) for the whole member.
"""
from __future__ import annotations

import copy

import numpy as np

from .abi import heat_flux, wind_stress

# Row dimension and value kind of every grid array that depends on the mesh.
# row: "node" (M+1), "cell" (N+1), "edge" (NE+1), "he" (NCV+1), "hei" (NCV_I+1),
#      "obc" (IOBCN+1), "riv" (NUMQBC+1), "obcl" (a list of open-boundary numbers)
# val: None (data), or the index space the values point into.
_ARRAYS = {
    "VX": ("node", None), "VY": ("node", None), "H": ("node", None), "ART1": ("node", None),
    "ART2": ("node", None), "GRAV_N": ("node", None), "NN_HVC": ("node", None),
    "SITA_GD": ("node", None), "PHPN": ("node", None), "ISONB": ("node", None),
    "NTSN": ("node", None), "NTVE": ("node", None), "NBSN": ("node", "node"),
    "NBVE": ("node", "cell"), "NBVT": ("node", None),
    "DLTXTRIE": ("node", None), "DLTYTRIE": ("node", None), "DLTXECEC": ("node", None),
    "DLTYECEC": ("node", None), "DLTXNEC": ("node", None), "DLTYNEC": ("node", None),
    "Z": ("node", None), "ZZ": ("node", None), "DZ": ("node", None), "DZZ": ("node", None),
    "XC": ("cell", None), "YC": ("cell", None), "ART": ("cell", None), "H1": ("cell", None),
    "COR": ("cell", None), "GRAV_E": ("cell", None), "CC_HVC": ("cell", None),
    "CC_SPONGE": ("cell", None), "CC_Z0B": ("cell", None), "EPOR": ("cell", None),
    "IUCP": ("cell", None), "ALPHA": ("cell", None), "NV": ("cell", "node"),
    "NBE": ("cell", "cell"), "ISBCE": ("cell", None), "A1U": ("cell", None),
    "A2U": ("cell", None), "AW0": ("cell", None), "AWX": ("cell", None), "AWY": ("cell", None),
    "Z1": ("cell", None), "ZZ1": ("cell", None), "DZ1": ("cell", None), "DZZ1": ("cell", None),
    "IEC": ("edge", "cell"), "IENODE": ("edge", "node"), "ISBC": ("edge", None),
    "XIJC": ("edge", None), "YIJC": ("edge", None), "DLTXC": ("edge", None),
    "DLTYC": ("edge", None),
    "NIEC": ("he", "node"), "NTRG": ("he", "cell"), "DLTXE": ("he", None), "DLTYE": ("he", None),
    "XIJE": ("he", None), "YIJE": ("he", None),
    "DLTXNCVE": ("hei", None), "DLTYNCVE": ("hei", None),
    "I_OBC_N": ("obc", "node"), "TYPE_OBC": ("obc", None), "NEXT_OBC": ("obc", "node"),
    "NADJC_OBC": ("obc", None), "ADJC_OBC": ("obc", "cell"), "FLUXF_OBC": ("obc", None),
    "DLTN_OBC": ("obc", None), "NXOBC": ("obc", None), "NYOBC": ("obc", None),
    "OBC_LST1": ("obcl", "obc"), "OBC_LST2": ("obcl", "obc"),
    "INODEQ": ("riv", "node"), "ICELLQ": ("riv", "cell"), "N_ICELLQ": ("riv", "node"),
    "RDISQ": ("riv", None), "QAREA": ("riv", None), "ANGLEQ": ("riv", None),
    "VQDIST": ("riv", None),
}
_COUNT = {"node": "M", "cell": "N", "edge": "NE", "he": "NCV", "hei": "NCV_I", "obc": "IOBCN",
          "riv": "NUMQBC"}


def perturbed_members(base, n, seed=0, wind=0.2, tide=0.1, t_sigma=0.5):
    """n member specs of ``base``: {"wind_scale", "tide_scale", "t_offset"}."""
    rng = np.random.default_rng(seed)
    return [{"wind_scale": float(rng.uniform(1.0 - wind, 1.0 + wind)),
             "tide_scale": float(rng.uniform(1.0 - tide, 1.0 + tide)),
             "t_offset": float(rng.normal(0.0, t_sigma))} for _ in range(n)]


def member_case(base, spec):
    """The standalone case of one member (for checks against the union)."""
    c = dict(base)
    c["forcing"] = copy.deepcopy(base["forcing"])
    c["init"] = dict(base["init"])
    if c["forcing"].get("tide") is not None:
        c["forcing"]["tide"]["apt"] = c["forcing"]["tide"]["apt"] * spec["tide_scale"]
    ws = wind_stress(base)
    if ws is not None:
        # PSIMPLE_DRAG of the scaled wind speed
        w = base["forcing"]["wind"]
        if w["kind"] == "speed":
            from .cases import simple_drag
            M1 = base["grid"]["N"] + 1
            sx, sy = simple_drag(np.full(M1, w["u"] * spec["wind_scale"]),
                                 np.full(M1, w["v"] * spec["wind_scale"]))
        else:
            sx, sy = ws[0] * spec["wind_scale"] ** 2, ws[1] * spec["wind_scale"] ** 2
        sx[0] = 0.0
        sy[0] = 0.0
        c["forcing"]["wind"] = {"kind": "field", "sx": sx, "sy": sy}
    c["init"]["t_offset"] = np.full(base["grid"]["M"] + 1, spec["t_offset"])
    c["name"] = base["name"] + "-member"
    return c


def union_case(base, specs):
    """One case holding every member of ``specs`` as a disjoint copy of ``base``'s mesh."""
    g = base["grid"]
    nm = len(specs)
    from .grid import Grid
    u = Grid()
    for k, v in g.a.items():
        if k not in _ARRAYS:
            u[k] = v
    for k, (row, val) in _ARRAYS.items():
        if k not in g.a:
            continue
        a = np.asarray(g[k])
        if row == "obcl":
            n_o = g["IOBCN"]
            u[k] = np.concatenate([a + m * n_o for m in range(nm)]).astype(a.dtype)
            continue
        cnt = g[_COUNT[row]]
        body = a[1:cnt + 1]
        parts = [a[:1]]
        for m in range(nm):
            b = body.copy()
            if val is not None:
                off = m * g[_COUNT[val]]
                b = np.where(b > 0, b + off, b).astype(a.dtype)
            parts.append(b)
        u[k] = np.concatenate(parts, axis=0)
    for key in ("M", "N", "NE", "NCV", "NCV_I", "IOBCN", "NUMQBC"):
        u[key] = g[key] * nm
    fc = base["forcing"]
    f = {}
    tide = fc.get("tide")
    if tide is not None:
        f["tide"] = {"period": tide["period"],
                     "apt": np.concatenate([tide["apt"] * s["tide_scale"] for s in specs]),
                     "phai": np.concatenate([tide["phai"]] * nm),
                     "emean": np.concatenate([tide["emean"]] * nm)}
    else:
        f["tide"] = None
    for k in ("qdis", "tdis", "sdis"):
        f[k] = np.concatenate([np.asarray(fc[k])] * nm)
    if fc.get("wind") is not None:
        sx = [np.zeros(1)]
        sy = [np.zeros(1)]
        for s in specs:
            ws = wind_stress(member_case(base, s))
            sx.append(ws[0][1:])
            sy.append(ws[1][1:])
        f["wind"] = {"kind": "field", "sx": np.concatenate(sx), "sy": np.concatenate(sy)}
    else:
        f["wind"] = None
    hf = heat_flux(base)
    if hf is not None:
        f["heat"] = {"swrad": np.concatenate([hf[0][:1]] + [hf[0][1:]] * nm),
                     "wtsurf": np.concatenate([hf[1][:1]] + [hf[1][1:]] * nm)}
    init = dict(base["init"])
    M = g["M"]
    toff = np.zeros(M * nm + 1)
    for m, s in enumerate(specs):
        toff[1 + m * M:1 + (m + 1) * M] = s["t_offset"]
    init["t_offset"] = toff
    return {"grid": u, "forcing": f, "params": base["params"], "init": init,
            "name": "%s-x%d" % (base["name"], nm), "members": nm, "member_grid": g}


def member_slice(union, m, name, engine):
    """Member m's part of field ``name`` of a union model, in the standalone layout."""
    g = union["member_grid"]
    a = engine.get(name)
    KB = engine.KB
    for cnt_key in ("M", "N"):
        cnt = g[cnt_key]
        total = cnt * union["members"] + 1
        if a.size == total:
            return np.concatenate([a[:1], a[1 + m * cnt:1 + (m + 1) * cnt]])
        if a.size == total * KB:
            a2 = a.reshape((total, KB), order="F")
            return np.concatenate([a2[:1], a2[1 + m * cnt:1 + (m + 1) * cnt]]).reshape(-1, order="F")
    raise KeyError("%s is not a node or cell field" % name)
