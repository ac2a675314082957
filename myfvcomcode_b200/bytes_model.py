"""Algorithmic (compulsory) HBM traffic of each kernel group of one internal step.

The ledger counts every array a kernel reads as read once and every array it writes as
written once per launch, at the storage width the library uses (FP64 fields, int32
indices and flags), with the mesh metrics, gather lists and 2-D fields included.  It is
the denominator-free byte count behind ``roofline.achieved``: achieved GB/s of a kernel =
ledger bytes of one launch / measured duration of one launch.  Re-reads through L1/L2 of
neighbour values (the gathers) are not compulsory and are not counted.

Sizes: M nodes, N cells, NE element edges, NCV = 3N control-volume half-edges,
K = KBM1 layers, KB = K+1 levels, S = ISPLIT, ring sizes from the mesh (sum of NTSN and
NTVE over nodes).
"""
from __future__ import annotations

D = 8   # FP64
I = 4   # int32


def sizes(grid):
    return dict(M=grid["M"], N=grid["N"], NE=grid["NE"], NCV=grid["NCV"], KB=grid["KB"],
                K=grid["KB"] - 1, ntsn=int(grid["NTSN"][1:].sum()), ntve=int(grid["NTVE"][1:].sum()))


def ledger(grid, isplit, wet_dry):
    """{group: (bytes per launch, launches per internal step)}"""
    s = sizes(grid)
    M, N, NE, NCV, K, KB = s["M"], s["N"], s["NE"], s["NCV"], s["K"], s["KB"]
    ntsn, ntve = s["ntsn"], s["ntve"]
    st = 4 * isplit
    ring = I * ntsn + 2 * D * ntsn          # NBSN + DLTXTRIE/DLTYTRIE entries
    halfedge_csr = I * 2 * NCV + I * (M + 1)
    halfedge_geo = NCV * (I + 2 * D) + NCV * (2 * I + 4 * D)  # NTRG, DLTXE/YE, NIEC, DLTXNCVE/YNCVE
    edge_geo = NE * (4 * I + I + 4 * D)     # IEC, IENODE, ISBC, XIJC/YIJC/DLTXC/DLTYC
    cell_lsq = N * (3 * I + 8 * D + 3 * I)  # NBE, A1U/A2U, CELL_EDGE
    g = {}
    # ---- external mode, per RK stage ----
    g["ext_node"] = (M * (I + I + 3 * D) + halfedge_csr + NCV * (I + 2 * D) + N * 3 * D, st)
    g["ext_cell"] = (N * (cell_lsq // N + 26 * D + 6 * I) + N * 8 * D + edge_geo + M * 4 * D, st)
    g["ext_update"] = (M * (6 * D + I) + N * (10 * D + (2 * I if wet_dry else 0)), st)
    if wet_dry:
        g["wet_judge"] = (N * (3 * I + I + D) + M * (4 * D + 2 * I) + I * ntve, st)
    # ---- 3-D, once per internal step ----
    g["cell_pre"] = (N * K * 4 * D + N * K * D + N * 12 * D, 1)              # U,V rw; DZ1; 2-D
    g["advection3d"] = (N * K * 4 * D + M * K * D + cell_lsq + N * 10 * D + edge_geo + M * D, 1)
    g["baropg"] = (M * K * 2 * D + N * KB * 2 * D + N * K * 7 * D + N * 10 * D + M * 3 * D, 1)
    g["int_advave"] = (N * (cell_lsq // N + 20 * D) + edge_geo + M * 3 * D, 1)
    g["adjust2"] = (N * K * 5 * D + N * 6 * D, 1)
    g["vertvl_flux"] = (N * K * 3 * D + M * K * D + halfedge_csr + NCV * (I + 2 * D) + N * D, 1)
    g["vertvl_col"] = (M * K * 2 * D + M * KB * D + M * K * 2 * D + M * 10 * D + I * ntve + N * 2 * D, 1)
    g["w_viscofh"] = (M * KB * D + N * KB * D + N * K * 2 * D + M * K * D + M * 3 * D
                      + ntve * (I + 4 * D) + N * I, 1)
    g["adv_uv"] = (N * K * 9 * D + N * D + M * K * D + cell_lsq + N * 14 * D + edge_geo + M * 2 * D, 1)
    g["vdif_uv"] = (N * KB * D + N * K * 10 * D + N * 20 * D + M * 3 * D, 1)
    g["grad_q"] = (M * K * 2 * D + M * K * 12 * D + ring + M * 2 * D, 1)
    g["adv_q"] = (M * K * (12 * D + 6 * D + 2 * D) + N * K * 4 * D + halfedge_csr + halfedge_geo
                  + M * 6 * D, 1)
    g["vdif_q"] = (M * KB * 14 * D + N * K * 2 * D + N * 4 * D + I * ntve + M * 6 * D, 1)
    g["grad_ts"] = (M * K * 4 * D + M * K * 12 * D + ring + M * 8 * D, 1)
    g["adv_ts"] = (M * K * (12 * D + 6 * D + 2 * D) + N * K * 3 * D + halfedge_csr + halfedge_geo
                   + M * 6 * D, 1)
    g["vdif_ts"] = (M * K * 5 * D + M * 12 * D, 1)
    g["bcond_ts"] = (grid["IOBCN"] * K * 8 * D, 1)
    g["final"] = (M * KB * 6 * D + N * KB * 7 * D + N * 6 * D + M * 4 * D, 1)
    return g


def step_bytes(grid, isplit, wet_dry):
    return sum(b * n for b, n in ledger(grid, isplit, wet_dry).values())
