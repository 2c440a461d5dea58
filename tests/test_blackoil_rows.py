"""The device path's three-phase residual and Jacobian rows against the oracle's assembly, on the CPU.

The kernels k_cells3 / k_perfs3 / k_wells3 run the __host__ __device__ row functions of
ressim_b200/csrc/rf_blackoil_rows.cuh once per cell, perforation and well.  Here the same source is
compiled for the host (tests/native/rows_host.cpp, g++ with -ffp-contract=off like the oracle), so
the port of the black-oil physics (PVT table with undersaturated branches, Stone II, gas-oil Pc,
the flash of undersaturated cells above the saturated Rs, gravity, gas and water injection) and
its assembly glue (neighbour order, signs, the triplet summation order) are checked against the
oracle's residual and Jacobian with no GPU.  On the GPU, the same rows run with CUDA's exp/pow,
so device results differ from these by rounding only.
"""
import ctypes as C
import math
import os
import subprocess

import numpy as np
import pytest

from oracle.oracle_py import OracleSimulator
from ressim_b200 import decks
from ressim_b200.pvt import PvtTable

HERE = os.path.dirname(os.path.abspath(__file__))
KDARCY = 8.5269888e-3


@pytest.fixture(scope="module")
def host(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("rows") / "rows_host.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-Wno-unknown-pragmas",
                    "-o", out, os.path.join(HERE, "native", "rows_host.cpp")], check=True)
    return C.CDLL(out)


def _p(a, t=C.c_double):
    return a.ctypes.data_as(C.POINTER(t))


def _geometry(d, abi):
    nx, ny, nz = d.nx, d.ny, d.nz
    n = nx * ny * nz
    kx, ky, kz = (np.asarray(a, dtype=float) for a in (d.perm_x, d.perm_y, d.perm_z))
    dz = np.asarray(d.dz, dtype=float)
    dx, dy = abi.dx, abi.dy
    tx, ty, tz = np.zeros(n), np.zeros(n), np.zeros(n)

    def harm(a, b):
        return 0.0 if a + b == 0.0 else 2.0 * a * b / (a + b)
    for i in range(n):
        ci, cj, ck = i % nx, (i // nx) % ny, i // (nx * ny)
        if ci + 1 < nx:
            tx[i] = KDARCY * (harm(kx[i], kx[i + 1]) * (dy * dz[ck]) / dx)
        if cj + 1 < ny:
            ty[i] = KDARCY * (harm(ky[i], ky[i + nx]) * (dx * dz[ck]) / dy)
        if ck + 1 < nz:
            p1, p2 = kz[i], kz[i + nx * ny]
            den = p2 * dz[ck] + p1 * dz[ck + 1]
            tz[i] = 0.0 if den <= 0.0 else KDARCY * (2.0 * p1 * p2 * (dx * dy) / den)
    pv = np.array([dx * dy * dz[i // (nx * ny)] * d.porosity[i] for i in range(n)])
    depth = np.array([abi.depth_reference_m + sum(dz[:k]) + dz[k] * 0.5 for k in range(nz)])
    return tx, ty, tz, pv, depth


def _wells(d, abi):
    """Physical wells (grouped by id in first-appearance order), one perforation per entry, the
    Peaceman index and each well's control (no schedules in these decks)."""
    groups, perf_well, perf_cell, perf_inj, has_wi, wi = {}, [], [], [], [], []
    for e, w in enumerate(d.wells):
        g = groups.setdefault(w.physical_well_id, len(groups))
        perf_well.append(g)
        cell = w.k * d.nx * d.ny + w.j * d.nx + w.i
        perf_cell.append(cell)
        perf_inj.append(int(w.injector))
        kx, ky = d.perm_x[cell], d.perm_y[cell]
        r_eq = 0.28 * math.sqrt(math.sqrt(kx / ky) * abi.dx ** 2 + math.sqrt(ky / kx) * abi.dy ** 2) / (
            (kx / ky) ** 0.25 + (ky / kx) ** 0.25)
        wi.append(KDARCY * 2.0 * math.pi * math.sqrt(kx * ky) * d.dz[w.k] / (math.log(r_eq / w.well_radius) + w.skin))
        has_wi.append(1)
    nw = len(groups)
    well_ptr, well_perfs, ctrl = [0], [], []
    for g in range(nw):
        ks = [k for k in range(len(perf_well)) if perf_well[k] == g]
        well_perfs += ks
        well_ptr.append(len(well_perfs))
        rep = d.wells[ks[0]]
        inj = bool(rep.injector)
        rate = (abi.injector_rate_controlled and abi.injector_enabled) if inj else abi.producer_rate_controlled
        surf = abi.target_injector_surface_rate_m3_day if inj else abi.target_producer_surface_rate_m3_day
        tgt = abi.target_injector_rate_m3_day if inj else abi.target_producer_rate_m3_day
        uses_surf = not math.isnan(surf)
        target = max(surf if uses_surf else tgt, 0.0) if rate else 0.0
        limit = abi.well_bhp_max if inj else abi.well_bhp_min
        ctrl += [1.0, float(bool(rate)), float(uses_surf), float(bool(rate)), float(inj), target, limit, rep.bhp]
    i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)  # noqa: E731
    return (nw, len(perf_well), i32(perf_cell), i32(perf_inj), i32(perf_well), i32(has_wi), np.array(wi),
            i32(well_ptr), i32(well_perfs), np.array(ctrl))


def _device_rows(host, d, dt, prev, cur, reg, bhp, q, heads):
    base = np.ascontiguousarray(d.rs, dtype=float)  # the DRSDT0 cap: the simulator's Rs
    abi, keep = d.to_abi()
    n = d.n_cells
    tx, ty, tz, pv, depth = _geometry(d, abi)
    nw, npf, pcell, pinj, pwell, phas, pwi, wptr, wperfs, ctrl = _wells(d, abi)
    N = 3 * n + nw + npf
    res = np.zeros(N)
    blocks = np.zeros(63 * n)
    jrw, jwr_perf, jwr_ctrl = np.zeros(3 * npf), np.zeros(3 * npf), np.zeros(3 * npf)
    jww_perf_bhp, jww_ctrl_q, jww_ctrl_bhp = np.zeros(npf), np.zeros(npf), np.zeros(nw)
    head = np.ascontiguousarray(heads, dtype=float)
    prev_, cur_ = (np.ascontiguousarray(a, dtype=float).ravel() for a in (prev, cur))
    reg_ = np.ascontiguousarray(reg, dtype=np.int32)
    rc = host.rfh_assemble3(C.byref(abi), C.c_double(dt), _p(tx), _p(ty), _p(tz), _p(pv), _p(depth),
                            _p(reg_, C.c_int32), _p(prev_), _p(cur_), nw, npf, _p(pcell, C.c_int32),
                            _p(pinj, C.c_int32), _p(pwell, C.c_int32), _p(phas, C.c_int32), _p(pwi), _p(head),
                            _p(wptr, C.c_int32), _p(wperfs, C.c_int32), _p(ctrl), _p(np.ascontiguousarray(bhp)),
                            _p(np.ascontiguousarray(q)), _p(res), _p(blocks), _p(jrw), _p(jwr_perf),
                            _p(jww_perf_bhp), _p(jwr_ctrl), _p(jww_ctrl_q), _p(jww_ctrl_bhp), _p(base))
    assert rc == 0
    J = np.zeros((N, N))
    nx, ny, nz = d.nx, d.ny, d.nz
    for i in range(n):
        ci, cj, ck = i % nx, (i // nx) % ny, i // (nx * ny)
        nbr = [i - nx * ny if ck > 0 else -1, i - nx if cj > 0 else -1, i - 1 if ci > 0 else -1, i,
               i + 1 if ci + 1 < nx else -1, i + nx if cj + 1 < ny else -1, i + nx * ny if ck + 1 < nz else -1]
        for s, j in enumerate(nbr):
            if j >= 0:
                J[3 * i:3 * i + 3, 3 * j:3 * j + 3] += blocks[(7 * i + s) * 9:(7 * i + s) * 9 + 9].reshape(3, 3)
    for k in range(npf):
        c, w, qo = pcell[k], pwell[k], 3 * n + nw + k
        J[3 * c:3 * c + 3, qo] = jrw[3 * k:3 * k + 3]
        J[qo, qo] = 1.0
        J[qo, 3 * c:3 * c + 3] = jwr_perf[3 * k:3 * k + 3]
        J[qo, 3 * n + w] = jww_perf_bhp[k]
    for w in range(nw):
        bo = 3 * n + w
        J[bo, bo] = jww_ctrl_bhp[w]
        for a in range(wptr[w], wptr[w + 1]):
            k = wperfs[a]
            J[bo, 3 * pcell[k]:3 * pcell[k] + 3] = jwr_ctrl[3 * k:3 * k + 3]
            J[bo, 3 * n + nw + k] = jww_ctrl_q[k]
    return res, J


def _state(d, seed):
    """Saturated cells with free gas, undersaturated cells below the saturated Rs, and
    undersaturated cells above it (they flash free gas inside the properties)."""
    n = d.n_cells
    rng = np.random.default_rng(seed)
    p = rng.uniform(150.0, 260.0, n)
    sw = rng.uniform(0.12, 0.45, n)
    reg = np.array([(i // 2) % 2 for i in range(n)], dtype=np.int32)
    table = PvtTable(d.pvt_rows, d.pvt_c_o)
    hc = np.where(reg == 0, rng.uniform(0.0, 0.2, n), 0.0)
    for i in range(n):
        if reg[i] == 1:
            hc[i] = table.interpolate(p[i]).rs_m3m3 * (0.7 if i % 3 else 1.04)
    cur = np.stack([p, sw, hc], axis=1)
    prev = cur.copy()
    prev[:, 0] += rng.uniform(-4.0, 4.0, n)
    prev[:, 1] += rng.uniform(-0.01, 0.01, n)
    return cur, prev, reg


def _drsdt0(d, seed):
    """Gas redissolution off, with each cell's Rs (the cap) below the saturated Rs at its pressure
    in many cells, so that the cap binds in the flash, the regimes and the properties."""
    d.set_gas_redissolution_enabled(False)
    table = PvtTable(d.pvt_rows, d.pvt_c_o)
    rng = np.random.default_rng(seed)
    d.rs = np.array([table.interpolate(float(p)).rs_m3m3 for p in d.pressure]) * rng.uniform(0.6, 1.0, d.n_cells)
    return d


def _tables(d):
    """SWOF/SGOF tables whose curves differ from the deck's Corey ones (exponents 2.5 / 1.8 and
    1.7 / 2.2), with knots the test states land on both sides of."""
    sw = np.array([0.1, 0.2, 0.3, 0.45, 0.6, 0.75, 0.9, 1.0])
    swof = np.stack([sw, np.clip((sw - 0.1) / 0.8, 0, 1) ** 2.5, np.clip((0.9 - sw) / 0.8, 0, 1) ** 1.8], axis=1)
    sg = np.array([0.0, 0.05, 0.15, 0.3, 0.5, 0.7, 0.85])
    sgof = np.stack([sg, np.clip((sg - 0.05) / 0.8, 0, 1) ** 1.7, np.clip((0.75 - sg) / 0.75, 0, 1) ** 2.2], axis=1)
    d.set_three_phase_scal_tables(swof, sgof)
    return d


@pytest.mark.parametrize("pc_og, fluid, gravity, drsdt0, tables",
                         [(False, "water", True, False, False), (True, "gas", True, False, False),
                          (True, "water", False, False, False), (False, "water", True, True, False),
                          (True, "gas", True, True, False), (False, "water", True, False, True),
                          (True, "gas", True, True, True)])
def test_blackoil_rows_match_oracle_assembly(host, pc_og, fluid, gravity, drsdt0, tables):
    d = decks.black_oil_3d(4, 3, 3, seed=3, dz=4.0, pc_og=pc_og, injected_fluid=fluid, rate_per_perf=8.0,
                           gravity=gravity)
    if drsdt0:
        d = _drsdt0(d, 21)
    if tables:
        d = _tables(d)
    cur, prev, reg = _state(d, seed=5)
    sim = OracleSimulator(d)
    nw, npf = sim.topology()
    rng = np.random.default_rng(9)
    bhp = np.array([170.0, 260.0, 240.0, 255.0, 140.0])[:nw]
    q = np.array([(-1.0 if w.injector else 1.0) * rng.uniform(2.0, 15.0) for w in d.wells])
    res_o, ptr_, col, val = sim.assemble_state_regimes(0.7, prev, cur, reg, reg, bhp, q)
    heads = sim.head_offsets()
    J_o = np.zeros((len(res_o), len(res_o)))
    for r in range(len(res_o)):
        J_o[r, col[ptr_[r]:ptr_[r + 1]]] += val[ptr_[r]:ptr_[r + 1]]
    res_d, J_d = _device_rows(host, d, 0.7, prev, cur, reg, bhp, q, heads)
    assert res_d.shape == res_o.shape
    rscale = np.maximum(np.abs(res_o), 1e-6 * np.max(np.abs(res_o)) + 1e-30)
    assert np.max(np.abs(res_d - res_o) / rscale) < 1e-12
    jscale = np.max(np.abs(J_o), axis=1, keepdims=True) + 1e-30
    err = np.abs(J_d - J_o) / jscale
    r, c = np.unravel_index(np.argmax(err), err.shape)
    assert err[r, c] < 1e-12, (r, c, J_d[r, c], J_o[r, c])
    sim.close()


def test_blackoil_derive_and_classify_match_oracle(host):
    """The device write-back flash (derive_cell3) and the substep-start classification against
    the oracle's probes (modes 4 and 6)."""
    from oracle.oracle_py import blackoil_probe

    d = decks.black_oil_3d(4, 3, 3, seed=3)
    abi, keep = d.to_abi()
    cur, _, reg = _state(d, seed=11)
    n = d.n_cells
    p, sw, hc = (np.ascontiguousarray(cur[:, k]) for k in range(3))
    out = np.zeros(6 * n)
    base = np.ascontiguousarray(d.rs, dtype=float)
    assert host.rfh_derive3(C.byref(abi), n, _p(p), _p(sw), _p(hc), _p(reg, C.c_int32), _p(base), _p(out)) == 0
    rows = np.asarray(d.pvt_rows, dtype=float)
    for i in range(n):
        o = blackoil_probe(rows, d.pvt_c_o, 6, [p[i], sw[i], hc[i], reg[i]])
        np.testing.assert_array_equal(out[6 * i:6 * i + 4], o[:4])
    sg = np.where(np.arange(n) % 3 == 0, 0.05, 0.0)
    rs = np.array([PvtTable(d.pvt_rows, d.pvt_c_o).interpolate(p[i]).rs_m3m3 * (0.9 if i % 2 else 1.0)
                   for i in range(n)])
    got = np.zeros(n, dtype=np.int32)
    assert host.rfh_classify3(C.byref(abi), n, _p(p), _p(sg), _p(np.ascontiguousarray(rs)), _p(base),
                              _p(got, C.c_int32)) == 0
    for i in range(n):
        o = blackoil_probe(rows, d.pvt_c_o, 4, [p[i], sw[i], sg[i], rs[i]])
        assert got[i] == int(o[0]), i
