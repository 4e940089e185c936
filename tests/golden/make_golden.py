"""Generate the golden fixtures of tests/golden/ from the reference's own kernels.

Runs the reference's HiPIMS kernels compiled for the host (oracle/_ref, built
from the reference sources by oracle/build_ref.py) under the reference's step
order, on small seeded cases, and stores inputs and outputs as .npz.  The
fixtures pin the CPU restatement (oracle/hipims_oracle.c) where oracle/_ref is
not available, e.g. on a machine without the reference tree.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "chans-hipims-flamegpu_b200"))

from hipims_b200 import scenarios as S  # noqa: E402
from hipims_b200.topology import boundary_codes  # noqa: E402
from oracle import oracle as O  # noqa: E402

KEYS = ("mask", "z", "h", "qx", "qy", "wl", "landuse", "rain_mask")


def mixed_bc_case(seed: int, order: int) -> dict:
    """20 x 24 valid cells, bumpy bed, wet/dry mix, every boundary type."""
    rng = np.random.default_rng(seed)
    ny, nx = 20, 24
    nodata = np.zeros((ny + 2, nx + 2), dtype=bool)
    nodata[0, :] = nodata[-1, :] = nodata[:, 0] = nodata[:, -1] = True
    nodata[8:11, 10:13] = True  # an interior hole
    types = [3, 4, 6, 7, 8] + ([9] if order == 1 else [])
    boxes = [(0, ny + 2, 0, 2, 6), (0, ny + 2, nx, nx + 2, 5), (0, 2, 2, 9, 3),
             (0, 2, 9, 16, 7), (ny, ny + 2, 2, 12, 8), (ny, ny + 2, 12, nx, 4)]
    if order == 1:
        boxes.append((0, 2, 16, nx, 9))
    mask = boundary_codes(nodata, default_bc=50, boxes=boxes)
    z = rng.uniform(0.0, 0.3, mask.shape) + np.linspace(0.0, 0.2, mask.shape[1])[None, :]
    h = np.where(rng.uniform(size=mask.shape) < 0.7, rng.uniform(0.0, 0.4, mask.shape), 0.0)
    h[:, : mask.shape[1] // 3] += 0.3
    qx = rng.normal(0.0, 0.05, mask.shape) * (h > 0)
    qy = rng.normal(0.0, 0.05, mask.shape) * (h > 0)
    h[nodata] = qx[nodata] = qy[nodata] = 0.0
    landuse = (rng.uniform(size=mask.shape) < 0.4).astype(np.uint8)
    rain_mask = (rng.uniform(size=mask.shape) < 0.5).astype(np.int16)
    return dict(mask=mask, z=z, h=h, qx=qx, qy=qy, wl=z + h, landuse=landuse,
                rain_mask=rain_mask, manning=[0.02, 0.05], dx=0.5, cfl=0.5, first_dt=1.0e-3,
                rain=np.array([[0.0, 1e-4, 2e-4], [1.0, 3e-4, 0.0], [5.0, 0.0, 1e-4]]),
                given_depth=np.array([[0.0, 0.3], [0.5, 0.45], [100.0, 0.2]]),
                given_wl=np.array([[0.0, 0.6], [100.0, 0.7]]),
                given_q=np.array([[0.0, 0.05, 0.01], [1.0, 0.1, -0.02], [100.0, 0.0, 0.0]]),
                export_step=0.75, steps=60, types=np.array(types))


def edge_case(name: str) -> dict:
    """Small and degenerate catchments, all boundaries RIGID (type 3) unless
    noted, bumpy bed (0-5 cm), 40 steps, export clip every 0.25 s:
      tiny3x5    3 x 5 cells (smaller than a tile), one wet cell in the middle
      row1x40    a single row, dam break along it
      col40x1    a single column, dam break along it (the RIGID ghost keeps
                 the normal momentum on north/south faces, so water crosses
                 the column's end walls, as in the reference)
      dry        20 x 30 OPEN ring, no water, no rain: dt grows tenfold per
                 step to the export clip
      late_rain  the dry case with rain from t = 0.06 s"""
    ny, nx, bc, wet, rain = {
        "tiny3x5": (3, 5, 30, "column", None),
        "row1x40": (1, 40, 30, "dam", None),
        "col40x1": (40, 1, 30, "dam", None),
        "dry": (20, 30, 50, "none", None),
        "late_rain": (20, 30, 50, "none",
                      np.array([[0.0, 0.0], [0.05, 0.0], [0.06, 2e-3], [100.0, 2e-3]])),
    }[name]
    rng = np.random.default_rng(len(name))
    nodata = np.ones((ny + 2, nx + 2), dtype=bool)
    nodata[1:-1, 1:-1] = False
    mask = boundary_codes(nodata, default_bc=bc)
    z = rng.uniform(0.0, 0.05, mask.shape)
    h = np.zeros(mask.shape)
    if wet == "dam":
        r, c = np.meshgrid(np.arange(ny + 2), np.arange(nx + 2), indexing="ij")
        h[:] = np.where((c <= (nx + 1) // 2) & (r <= (ny + 1) // 2 + (ny == 1)), 0.6, 0.05)
    elif wet == "column":
        h[(ny + 2) // 2, (nx + 2) // 2] = 1.0
    h[nodata] = 0.0
    zeros = np.zeros(mask.shape)
    d = dict(mask=mask, z=z, h=h, qx=zeros.copy(), qy=zeros.copy(), wl=z + h,
             landuse=np.zeros(mask.shape, dtype=np.uint8), manning=[0.03], dx=1.0, cfl=0.5,
             first_dt=1.0e-4, export_step=0.25, steps=40)
    if rain is not None:
        d["rain"] = rain
    return d


EDGE_CASES = ("tiny3x5", "row1x40", "col40x1", "dry", "late_rain")


def cases() -> dict:
    out = {}
    for name in EDGE_CASES:
        for order in (1, 2):
            out[f"edge_{name}_o{order}"] = (edge_case(name), order)
    d = S.dam_break(48)
    d.update(steps=120)
    out["dam_break48_o2"] = (d, 2)
    out["dam_break48_o1"] = (dict(d), 1)
    c = S.channel()
    c.update(steps=100000)
    out["channel_o2"] = (c, 2)
    c1 = dict(c)
    c1["t_end"] = 2.0
    out["channel_o1"] = (c1, 1)
    out["mixed_bc_o2"] = (mixed_bc_case(11, 2), 2)
    out["mixed_bc_o1"] = (mixed_bc_case(12, 1), 1)
    u = S.urban_catchment(24, dx=2.0, seed=9)
    u.update(steps=200, infiltration=dict(ks=[2.0e-6, 5.0e-6], psi=[0.11, 0.2],
                                          dtheta=[0.3, 0.45]))
    out["urban24_infil_o2"] = (u, 2)
    return out


def run_case(d: dict, order: int, backend: str) -> tuple[dict, int]:
    sim = O.Sim(d, order=order, backend=backend, export_step=d.get("export_step", 1.0e30))
    n = sim.run(int(d["steps"]), float(d.get("t_end", np.inf)))
    st = sim.state()
    st["steps"] = n
    st["exports"] = sim.g.exports
    return st, n


def main() -> None:
    if not O.ref_available():
        raise SystemExit("oracle/_ref is not built: python oracle/build_ref.py")
    only = set(sys.argv[1:])
    for name, (d, order) in cases().items():
        if only and name not in only:
            continue
        st, n = run_case(d, order, "ref")
        payload = {k: np.asarray(d[k]) for k in KEYS if d.get(k) is not None}
        for k in ("manning", "rain", "given_depth", "given_wl", "given_q"):
            if d.get(k) is not None:
                payload[k] = np.asarray(d[k], dtype=np.float64)
        scal = dict(dx=d["dx"], cfl=d["cfl"], first_dt=d["first_dt"], order=order,
                    steps=d["steps"], t_end=d.get("t_end", np.inf),
                    export_step=d.get("export_step", 1.0e30))
        for k, v in scal.items():
            payload["in_" + k] = np.asarray(v, dtype=np.float64)
        if d.get("infiltration") is not None:
            for k in ("ks", "psi", "dtheta"):
                payload["infil_" + k] = np.asarray(d["infiltration"][k], dtype=np.float64)
        for k in ("h", "qx", "qy", "wl", "h_max", "cum"):
            if k in st:
                payload["out_" + k] = st[k]
        payload["out_t"] = np.asarray(st["t"])
        payload["out_dt"] = np.asarray(st["dt"])
        payload["out_steps"] = np.asarray(n)
        payload["out_exports"] = np.asarray(st["exports"])
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **payload)
        print(f"{name}: {n} steps, t={st['t']:.6f}, -> {os.path.getsize(path)} bytes")


def load_case(path: str) -> tuple[dict, int, dict]:
    """Inverse of main(): (inputs dict for oracle.Sim, order, expected outputs)."""
    z = np.load(path)
    d = {k: z[k] for k in KEYS if k in z.files}
    for k in ("manning", "rain", "given_depth", "given_wl", "given_q"):
        if k in z.files:
            d[k] = z[k]
    for k in ("dx", "cfl", "first_dt", "steps", "t_end", "export_step"):
        d[k] = float(z["in_" + k])
    d["steps"] = int(d["steps"])
    if "infil_ks" in z.files:
        d["infiltration"] = {k: z["infil_" + k] for k in ("ks", "psi", "dtheta")}
    order = int(z["in_order"])
    exp = {k[4:]: z[k] for k in z.files if k.startswith("out_")}
    return d, order, exp


if __name__ == "__main__":
    main()
