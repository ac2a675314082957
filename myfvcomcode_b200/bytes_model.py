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


def ledger(grid, isplit, wet_dry, precision="fp64", compact=False):
    """{group: (bytes per launch, launches per internal step)}

    ``precision`` "fp32flux" counts the arrays that form keeps in FP32 at 4 bytes: the
    least-squares and node-ring gradients (A1U/A2U, the 2-D and 3-D cell gradients,
    PTPX.. with the ring extrema), the edge offsets, DLTXC/DLTYC, ART, CC_HVC and the
    control-volume metrics read by the flux kernels.  FP64 state is counted at 8 bytes
    in both forms (ADVX/ADVY, UF/VF/VISCOFM and DZ1 among them).

    ``compact`` (precision form only): the Runge-Kutta stages' cell kernel is the compact
    one, whose records replace the slot table's metrics and EXTUV's fixed inputs (see
    ``ext_cell_compact``).
    """
    s = sizes(grid)
    M, N, NE, NCV, K, KB = s["M"], s["N"], s["NE"], s["NCV"], s["K"], s["KB"]
    ntsn, ntve = s["ntsn"], s["ntve"]
    X = 4 if precision == "fp32flux" else D  # width of the flux kernels' scratch and metrics
    st = 4 * isplit
    ring = I * ntsn + 2 * D * ntsn          # NBSN + DLTXTRIE/DLTYTRIE entries
    halfedge_csr = I * 2 * NCV + I * (M + 1)
    halfedge_geo = NCV * (I + 2 * X) + NCV * (2 * I + 4 * X)  # NTRG, DLTXE/YE, NIEC, DLTXNCVE/YNCVE
    # IEC, IENODE, ISBC, and the edge offsets (XIJC/YIJC with XC/YC) and DLTXC/DLTYC
    edge_off = NE * 2 * D + N * 2 * D if X == D else NE * 4 * X
    edge_geo = NE * (4 * I + I + 2 * X) + edge_off
    cell_lsq = N * (3 * I + 8 * X + 3 * I)  # NBE, A1U/A2U, CELL_EDGE
    pg_extra = 0 if X == D else NE * 2 * D  # FP64 DLTXC/DLTYC of the surface-slope term
    g = {}
    # ---- external mode, per RK stage ----
    # The update after each stage (external_step.F:333-436) runs inside the next stage's
    # kernels: its node part (ELF read, H read, EL, D, DTFA written) at the head of
    # k_ext_node, its cell part (H1 read, EL1, D1 and the three half-edge continuity
    # fluxes written, CELL_HE read) at the tail of k_ext_cell; one closing launch
    # (k_ext_finish) does the last stage's node part and the UA/VA copies.
    # With wetting and drying WET_JUDGE's node part (ELF read and written, H read, ISWETN
    # written, the NBVE ring of cell flags) also runs at the head of k_ext_node; its cell
    # part (the three nodes' ELF and H, ISWETC and ELF1 written) keeps its own kernel.
    wet_node = (M * (3 * D + 2 * I) + I * ntve) if wet_dry else 0
    g["ext_node"] = (M * (I + I + 3 * D) + halfedge_csr + NCV * (I + 2 * D) + N * 3 * D + M * 5 * D + wet_node, st)
    g["ext_cell"] = (N * (cell_lsq // N + 22 * D + 4 * X + 6 * I) + N * 8 * D + edge_geo + pg_extra
                     + M * 4 * D + N * (6 * D + 3 * I), st)
    if compact and precision == "fp32flux":
        g["ext_cell"] = (ext_cell_compact(N, M, isplit), st)
    g["ext_update"] = (M * (6 * D + I) + N * (10 * D + (2 * I if wet_dry else 0)), 1)
    if wet_dry:
        g["wet_judge"] = (N * (3 * I + I + D) + M * D, st)
    # ---- 3-D, once per internal step ----
    g["cell_pre"] = (N * K * 4 * D + N * K * D + N * 12 * D, 1)              # U,V rw; DZ1; 2-D
    # U, V read and ADVX, ADVY written per cell and layer (FP64 in both forms)
    g["advection3d"] = (N * K * 4 * D + M * K * D + cell_lsq + N * 6 * D + N * 4 * X
                        + edge_geo + M * D, 1)
    g["baropg"] = (M * K * 2 * D + N * KB * 2 * D + N * K * 7 * D + N * 10 * D + M * 3 * D, 1)
    g["int_advave"] = (N * (cell_lsq // N + 16 * D + 4 * X) + edge_geo + pg_extra + M * 3 * D, 1)
    # ADJUST2D3D(2) also writes VERTVL_EDGE's half-edge fluxes (CELL_HE, DLTXE/YE read
    # once per cell); the node kernel sums them in half-edge order.
    g["adjust2"] = (N * K * 5 * D + N * 6 * D + NCV * K * D + NCV * (I + 2 * D), 1)
    g["vertvl_flux"] = (NCV * K * D + M * K * D + halfedge_csr, 1)
    g["vertvl_col"] = (M * K * 2 * D + M * KB * D + M * K * 2 * D + M * 10 * D + I * ntve + N * 2 * D, 1)
    g["w_viscofh"] = (M * KB * D + N * KB * D + N * K * 2 * D + M * K * D + M * 3 * D
                      + ntve * (I + 4 * D) + N * I, 1)
    # U, V, W, DZ1, DRHOX, DRHOY read and UF, VF, VISCOFM written per cell and layer
    g["adv_uv"] = (N * K * 9 * D + N * D + M * K * D + cell_lsq + N * 10 * D + N * 4 * X
                   + edge_geo + M * 2 * D, 1)
    g["vdif_uv"] = (N * KB * D + N * K * 10 * D + N * 20 * D + M * 3 * D, 1)
    g["grad_q"] = (M * K * 2 * D + M * K * 12 * X + ring + M * 2 * D, 1)
    g["adv_q"] = (M * K * (12 * X + 6 * D + 2 * D) + N * K * 4 * D + halfedge_csr + halfedge_geo
                  + M * 6 * D, 1)
    g["vdif_q"] = (M * KB * 14 * D + N * K * 2 * D + N * 4 * D + I * ntve + M * 6 * D, 1)
    g["grad_ts"] = (M * K * 4 * D + M * K * 12 * X + ring + M * 8 * D, 1)
    g["adv_ts"] = (M * K * (12 * X + 6 * D + 2 * D) + N * K * 3 * D + halfedge_csr + halfedge_geo
                   + M * 6 * D, 1)
    g["vdif_ts"] = (M * K * 5 * D + M * 12 * D, 1)
    g["bcond_ts"] = (grid["IOBCN"] * K * 8 * D, 1)
    g["final"] = (M * KB * 6 * D + N * KB * 7 * D + N * 6 * D + M * 4 * D, 1)
    return g


def ext_cell_compact(N, M, isplit):
    """Bytes of one launch of the compact stage kernel, averaged over the 4*ISPLIT stages.

    Per cell: the flag word, UA, VA, the two wet flags, D1, the packed FP32 gradient
    {UX, UY, VX, VY}, {ART, CC_HVC} in FP32, {XC, YC}, three 16-byte slots, the two
    32-byte records of EXTUV's terms, UARK, VARK, ELRK1, ELF1 read; UAF, VAF, EL1, D1
    and the three half-edge continuity fluxes written.  Per node: {VX, VY}, D, EL read.
    The first stage of each external step also reads EL1 and writes UARK, VARK, ELRK1
    (instead of reading them); the last stage writes ADVUA, ADVVA, PSTX, PSTY.
    """
    per_cell = I + 2 * D + 2 * I + D + 16 + 8 + 16 + 3 * 16 + 2 * 32 + 4 * D + 4 * D + 3 * D
    st = 4 * isplit
    extra = (isplit * D + 4 * D) / st
    return int(N * (per_cell + extra) + M * (16 + 2 * D))


def step_bytes(grid, isplit, wet_dry, precision="fp64", compact=False):
    return sum(b * n for b, n in ledger(grid, isplit, wet_dry, precision, compact).values())
