"""The GPU matrix builder's candidate search, checked on the CPU at the full
benchmark geometry.

ctbb_icd_b200/csrc/ssm.cu builds the stored system matrix column-major: the
thread of a (column, view) cell evaluates only the channels and rows that a
conservative geometric bound admits (chan_of over the column's sampling
segments padded by 1 channel, 3 with a flying focal spot; row_range padded
by one row; every row near 45 degrees), each with the reference's exact
arithmetic. Its indices and weights equal the reference's wherever that
bound contains every (channel, row) whose ray reaches the column. This test
restates the bound (ssm.cu chan_of, row_range, ssm_cells_kernel) in numpy
and checks it against every entry the oracle's ray-driven builder (the
reference's loops, generate_system_matrix_ffs.cpp:60-239) produces for
sampled columns of the 512 x 512, 736 x 64, in-plane flying focal spot
geometry after load_raw's slice tables (table_direction -1), over every
view of the window.
"""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

import ctbb_icd_b200 as C  # noqa: E402
from ctbb_icd_b200 import workloads as W  # noqa: E402
import oracle_util as O  # noqa: E402


def view_tables(g, ffs):
    """Per-view source, frame and flying-focal-spot deflection (ssm.cu
    host_tables; generate_system_matrix.cpp:85-100, generate_system_matrix_ffs
    .cpp:66-67, 134, 242-290: in-plane +/-da e_u by view parity, z -/+dr e_w
    -/+dr tan(anode_angle) e_z with the angle in degrees passed to tan, or the
    four combinations of both)."""
    nvsm = int(g.num_views_for_system_matrix)
    i = np.arange(nvsm, dtype=np.float64)
    k = np.arange(nvsm)
    ta = (i - 0.5 * nvsm) * g.tube_angle_increment
    ew0, ew1, eu0, eu1 = np.cos(ta), np.sin(ta), -np.sin(ta), np.cos(ta)
    zs = g.table_direction * (i - 0.5 * nvsm) * g.tube_z_increment
    SDD, R = g.source_detector_distance, g.focal_spot_radius
    da = SDD * R * np.sin(g.fan_angle_increment) / (4.0 * (SDD - R))
    dr = SDD * g.CollSlicewidth / (4.0 * (SDD - R) * np.tan(g.anode_angle * 3.14159265359 / 180.0))
    a = np.zeros(nvsm)  # in-plane deflection along e_u
    r = np.zeros(nvsm)  # z-spot deflection along e_w (and r tan(anode_angle) along e_z)
    if ffs and not g.Zffs:
        a = np.where(k % 2 == 0, da, -da)
    elif ffs and not g.Phiffs:
        r = np.where(k % 2 == 0, -dr, dr)
    elif ffs:
        r = np.where(k % 4 < 2, -dr, dr)
        a = np.where(k % 2 == 0, -da, da)
    off0, off1, off2 = r * ew0 + a * eu0, r * ew1 + a * eu1, r * np.tan(g.anode_angle)
    return dict(src0=R * ew0 + off0, src1=R * ew1 + off1, src2=zs + off2, ew0=ew0, ew1=ew1, eu0=eu0, eu1=eu1,
                off0=off0, off1=off1, off2=off2)


def candidate_slack(g, ffs, col, v, ch, row):
    """For entries (view v, channel ch, row) of column `col`: how far each sits
    inside the builder's candidate channel range and row range (negative:
    outside, the entry would be missed)."""
    V = {k: a[v] for k, a in view_tables(g, ffs).items()}
    nx, nch, nr = int(g.num_voxels_x), int(g.n_channels), int(g.Nrows_projection)
    ic, jc = col % nx, col // nx
    vx, vy, vz = g.voxel_size_x, g.voxel_size_y, g.voxel_size_z
    xc, yc = (ic - g.center_voxel_x) * vx, (jc - g.center_voxel_y) * vy
    cc = g.center_channel_non_ffs
    dgam = g.fan_angle_increment if ffs else g.transaxial_detector_spacing / g.source_detector_distance

    def chan_of(px, py):
        rx, ry = px - V["src0"], py - V["src1"]
        a = -(rx * V["ew0"] + ry * V["ew1"])
        b = -(rx * V["eu0"] + ry * V["eu1"])
        return np.arctan2(b, a) / dgam + cc

    cs = np.stack([chan_of(xc, yc - vy), chan_of(xc, yc + vy), chan_of(xc - vx, yc), chan_of(xc + vx, yc)])
    pad = 3 if ffs else 1
    ch_lo = np.maximum(np.floor(cs.min(axis=0)).astype(np.int64) - pad, 0)
    ch_hi = np.minimum(np.ceil(cs.max(axis=0)).astype(np.int64) + pad, nch - 1)

    SDD = g.source_detector_distance
    tang = (ch - cc) * (g.fan_angle_increment if ffs else g.transaxial_detector_spacing / SDD)
    A, B = -SDD * np.cos(tang), SDD * np.sin(tang)
    D0 = (A * V["ew0"] - B * V["eu0"]) - V["off0"]
    D1 = (A * V["ew1"] - B * V["eu1"]) - V["off1"]
    ad0, ad1 = np.abs(D0), np.abs(D1)
    xmaj = ad0 > ad1
    D = np.where(xmaj, D0, D1)
    L = np.where(xmaj, xc - V["src0"], yc - V["src1"]) / D
    sa, cr = g.axial_detector_spacing, g.center_row
    with np.errstate(divide="ignore", invalid="ignore"):
        k0 = cr + (V["src2"] - vz) / (sa * L) - V["off2"] / sa
        k1 = cr + (V["src2"] + vz) / (sa * L) - V["off2"] / sa
    lo = np.floor(np.minimum(k0, k1)).astype(np.int64) - 1
    hi = np.ceil(np.maximum(k0, k1)).astype(np.int64) + 1
    all_rows = (np.abs(ad0 - ad1) <= 1e-9 * np.maximum(ad0, ad1)) | ~(np.abs(L) > 1e-12)
    r_lo = np.where(all_rows, 0, np.maximum(lo, 0))
    r_hi = np.where(all_rows, nr - 1, np.minimum(hi, nr - 1))
    return np.minimum.reduce([ch - ch_lo, ch_hi - ch, row - r_lo, r_hi - row])


# The benchmark geometries, and cfg2's scanner with the z flying focal spot
# (32 rows per projection, setup.cpp:225) alone and with the in-plane one.
CASES = {
    "cfg2": ("cfg2", None),
    "cfg1": ("cfg1", None),
    "cfg2_zffs": ("cfg2", {"Zffs": 1, "Phiffs": 0, "center_row": 15.5}),
    "cfg2_zphiffs": ("cfg2", {"Zffs": 1, "Phiffs": 1, "center_row": 15.5, "Readings": 18432}),
}


@pytest.mark.parametrize("case", list(CASES))
def test_candidate_bounds_contain_every_reference_entry_at_bench_size(tmp_path, case):
    name, overrides = CASES[case]
    _, rp = W.materialise(name, str(tmp_path), raw=False, overrides=overrides)
    C.slice_tables(rp)  # load_raw's tables set table_direction (setup.cpp:275)
    g = rp.geom
    assert g.table_direction == -1
    ffs = bool(g.Phiffs or g.Zffs)
    nx = int(g.num_voxels_x)
    ncol = nx * int(g.num_voxels_y)
    nvsm = int(g.num_views_for_system_matrix)
    per_view = int(g.n_channels) * int(g.Nrows_projection)
    rng = np.random.default_rng(2884)
    special = [nx // 2 + nx * (nx // 2), nx // 2 + nx * 3, 3 + nx * (nx // 2), nx // 4 + nx * (nx // 4),
               (3 * nx) // 4 + nx * (nx // 8)]
    cols = np.unique(np.concatenate([special, rng.integers(0, ncol, 16)])).astype(np.int64)
    ref = O.port_ssm_subset(rp, cols, np.arange(nvsm, dtype=np.int32))
    n_checked = 0
    for c in cols:
        q = ref[int(c)][0].astype(np.int64)
        if q.size == 0:
            continue
        v, rem = q // per_view, q % per_view
        ch, row = rem // int(g.Nrows_projection), rem % int(g.Nrows_projection)
        slack = candidate_slack(g, ffs, int(c), v, ch, row)
        assert slack.min() >= 0, (case, int(c), int(slack.min()), int(np.count_nonzero(slack < 0)))
        n_checked += q.size
    # Measured: every entry sits at least 3 channels inside its candidate
    # range and, away from the detector's first and last rows (where the
    # range is clamped), at least 2 rows inside.
    assert n_checked > 50000
