"""The optical bench after the transport: OBD and SideOBD on the GPU.

Drop-in for ``pymopt.optics.OBD`` / ``SideOBD`` / ``Grass``
(pymopt/optics/_classes.py:223-566): the same params keys and defaults,
``set_params``, ``set_monte_data``, ``load_file``, ``start``, ``get_result``
and ``save_result``. The result is the photodiode intensity for every
detector offset Z of the scan.

Per Z the exit photons pass through:
- lens 1;
- an annular slit;
- the laser-diode mount (optional);
- a second slit;
- lens 2.

The reference computes this with NumPy arrays, one Z at a time. Here
``pmo_run_obd`` traces every (photon, Z) pair in one kernel launch.

The Fresnel decision at each lens surface is random in the reference
(``np.random.rand() > R``). Here it uses Philox draws keyed by ``seed``. The
intensities agree with the reference statistically. With ``fixed_u`` set,
they agree photon by photon.
"""
from __future__ import annotations

import bz2
import ctypes as C
import json
import pickle

import numpy as np
import torch

from . import _abi as A
from . import engine as E
from ._lib import check, load
from .utils import set_params

__all__ = ["OBD", "SideOBD", "Grass"]


class Grass:
    """Glass refractive indices and the side geometry's angles
    (pymopt/optics/_classes.py:223-293)."""

    def __init__(self):
        self.supported_type = ["N-BK7", "N-SF11"]

    def get_inital_angle(self, slit_radius=10, lens_curvature_radius=51.68, wavelength=850,
                         grass_type="N-BK7"):
        n_1 = self.get_refractive_index(wavelength, grass_type)
        a1 = np.arcsin(slit_radius / lens_curvature_radius)
        a2 = np.arcsin(np.sin(a1) / n_1)
        return np.arcsin(n_1 * np.sin(a1 - a2))

    def get_real_bfl(self, slit_radius=10, lens_curvature_radius=51.68, lens_ct=10.,
                     wavelength=850, grass_type="N-BK7"):
        n_1 = self.get_refractive_index(wavelength, grass_type)
        a1 = np.arcsin(slit_radius / lens_curvature_radius)
        a2 = np.arcsin(np.sin(a1) / n_1)
        a3 = a1 - a2
        a4 = np.arcsin(n_1 * np.sin(a3))
        length = np.sqrt(lens_curvature_radius ** 2 - slit_radius ** 2) \
            - lens_curvature_radius + lens_ct
        dx = length * np.tan(a3)
        return (slit_radius - dx) / np.tan(a4)

    def get_refractive_index(self, ramda, grass_type="N-BK7"):
        n = 1.517
        if grass_type == "N-BK7":
            n = self._NBK7(ramda)
        if grass_type == "N-SF11":
            n = self._NSF11(ramda)
        return n

    # cubic fits of the catalogue indices against the wavelength in um
    # (pymopt/optics/_classes.py:268-293)
    def _NBK7(self, ramda):
        x = ramda * 1e-3
        if 312.6 <= ramda <= 486.1:
            return -2.4880 * x ** 3 + 3.5910 * x ** 2 - 1.8102 * x + 1.8395
        if 486.1 < ramda <= 852.1:
            return -0.1605 * x ** 3 + 0.3866 * x ** 2 - 0.3307 * x + 1.6102
        if 852.1 < ramda <= 2325:
            return -0.0029 * x ** 3 + 0.0125 * x ** 2 - 0.0304 * x + 1.5284
        raise ValueError("The wavelength is over the range that can be supported.")

    def _NSF11(self, ramda):
        x = ramda * 1e-3
        if 404.7 <= ramda <= 589.3:
            return -4.4506 * x ** 3 + 7.8207 * x ** 2 - 4.7512 * x + 2.7792
        if 589.3 < ramda <= 852.1:
            return -0.4659 * x ** 3 + 1.1864 * x ** 2 - 1.0622 * x + 2.0937
        if 852.1 < ramda <= 1060:
            return 0.0427 * x ** 2 - 0.1192 * x + 1.8324
        if 1060 < ramda <= 2325.4:
            return -0.0046 * x ** 3 + 0.0257 * x ** 2 - 0.0648 * x + 1.7993
        raise ValueError("The wavelength is over the range that can be supported.")


class OBD:
    """Optical bench of the reference (pymopt/optics/_classes.py:381-526).

    ``seed`` keys the Fresnel decisions (random when None); ``fixed_u`` in
    [0, 1) replaces every draw by that value (deterministic, for checks)."""

    def __init__(self, *, seed=None, fixed_u=None, device=None):
        self.params = {
            "start": -2.04, "end": 62.96, "split": 0.25, "wavelength": 850,
            "outerD_1": 50, "efl_1": 100, "bfl_1": 93.41,
            "ct_1": 10, "et_1": 3.553, "r_1": 51.68, "n_1": 1.517,
            "substrate_1": "N-BK7",
            "outerD_2": 50, "efl_2": 50, "bfl_2": 43.28,
            "ct_2": 12, "et_2": 3.01, "r_2": 39.24, "n_2": 1.758,
            "substrate_2": "N-SF11",
            "slit_outerD": 50, "slit_D": 20, "slit_width": 2, "slit_thickness": 5,
            "d_pd": 3,
            "ld_fix_part": True,
            "distance_2slits": 37, "pd_poit_correction": 0,
            "inversion": False, "side": False,
        }
        self._set_refrective_index()
        self.keys_params = list(self.params.keys())
        self.data = {"p": 0, "v": 0, "w": 0, "nPh": 1000, "z_max": 0}
        self.keys_data = list(self.data.keys())
        self.nPh = 1000
        self.seed = int(np.random.randint(2 ** 31)) if seed is None else int(seed)
        self.fixed_u = fixed_u
        self.device = device

    def _set_refrective_index(self):
        grass = Grass()
        self.params["n_1"] = grass.get_refractive_index(self.params["wavelength"],
                                                        self.params["substrate_1"])
        self.params["n_2"] = grass.get_refractive_index(self.params["wavelength"],
                                                        self.params["substrate_2"])

    def set_params(self, *initial_data, **kwargs):
        set_params(self.params, self.keys_params, *initial_data, **kwargs)
        self._set_refrective_index()

    def set_monte_data(self, *initial_data, **kwargs):
        set_params(self.data, self.keys_data, *initial_data, **kwargs)
        self.nPh = self.data["nPh"]

    def open_pklbz2_file(self, path):
        with bz2.open(path, "rb") as fp:
            return pickle.loads(fp.read())

    def open_jason_file(self, path):
        with open(path, "r") as fp:
            return json.load(fp)

    def load_file(self, path):
        self.data = self.open_pklbz2_file(path)
        self.nPh = self.data["nPh"]

    def start(self, show_graph=False):
        import pandas as pa
        res = self.opticalAnalysisMeth()
        if show_graph:
            raise NotImplementedError("plotting is not part of this package")
        self.result = pa.DataFrame(res, index=["Z", "int"]).T
        with np.errstate(divide="ignore"):
            self.result["log(int)"] = np.log10(res[1] / self.nPh)

    def get_result(self):
        return self.result

    def save_result(self, path):
        self.result.to_csv(path + "_opt.csv", index=False)

    # ---- the photons entering the bench (pymopt/optics/_classes.py:495-522)
    def _photons(self):
        if self.params["side"]:
            self.data["v"] = self.data["v"][[2, 1, 0]]
            self.data["p"] = self.data["p"][[2, 1, 0]]
            self.data["p"][0] -= self.params["side"] / 2
            self.data["p"][2] += self.params["side"] / 2
        v_all = self.data["v"]
        sel = v_all[2] > 0 if self.params["inversion"] else v_all[2] < 0
        p = self.data["p"][:, sel]
        p[2] = 0
        v = v_all[:, sel]
        if self.params["inversion"]:
            p[1] *= -1
            v[2] *= -1
            v[1] *= -1
        w = self.data["w"][sel]
        return p, v, w

    def _side_shift(self):
        return 0, 0.0, 0.0

    def opticalAnalysisMeth(self):
        """(Z, intensity) of the scan, traced on the GPU."""
        step = np.arange(self.params["start"], self.params["end"], self.params["split"])
        p, v, w = self._photons()
        dev = E.require_cuda(self.device)
        as_dev = lambda a: torch.from_numpy(  # noqa: E731
            np.ascontiguousarray(a, dtype=np.float32)).to(dev)
        dp_, dv, dw = as_dev(p), as_dev(v), as_dev(w)
        z = torch.from_numpy(np.ascontiguousarray(step, dtype=np.float64)).to(dev)
        out = torch.zeros(step.size, dtype=torch.float64, device=dev)
        side, side_dz, side_tan = self._side_shift()
        prm = self._struct(z, step.size, side, side_dz, side_tan)
        st = load().pmo_run_obd(C.byref(prm), dp_.data_ptr(), dv.data_ptr(), dw.data_ptr(),
                                int(dw.numel()), out.data_ptr(), E._stream_handle())
        check(st, "pmo_run_obd")
        return step, out.cpu().numpy()

    def _struct(self, z, n_z, side, side_dz, side_tan) -> A.PmoObdParams:
        P = self.params
        s = A.PmoObdParams()
        s.outer_d1, s.ct1, s.r1, s.n1, s.bfl1 = (float(P[k]) for k in
                                                 ("outerD_1", "ct_1", "r_1", "n_1", "bfl_1"))
        s.outer_d2, s.ct2, s.r2, s.n2, s.bfl2 = (float(P[k]) for k in
                                                 ("outerD_2", "ct_2", "r_2", "n_2", "bfl_2"))
        s.slit_d, s.slit_width = float(P["slit_D"]), float(P["slit_width"])
        s.slit_thickness, s.distance_2slits = float(P["slit_thickness"]), float(P["distance_2slits"])
        s.d_pd, s.pd_correction = float(P["d_pd"]), float(P["pd_poit_correction"])
        s.ld_fix_part = 1 if P["ld_fix_part"] else 0
        s.side, s.side_dz, s.side_tan = int(side), float(side_dz), float(side_tan)
        s.z, s.n_z = z.data_ptr(), int(n_z)
        s.seed = self.seed & 0xFFFFFFFFFFFFFFFF
        s.fixed_u = -1.0 if self.fixed_u is None else float(self.fixed_u)
        return s


class SideOBD(OBD):
    """The bench seen from the side (pymopt/optics/_classes.py:528-566): the
    photons' x is shifted by -(Z + dz) tan(theta0) at every Z."""

    def _photons(self):
        sel = self.data["v"][2] < 0
        p = self.data["p"][:, sel]
        p[2] = 0
        return p, self.data["v"][:, sel], self.data["w"][sel]

    def _side_shift(self):
        grass = Grass()
        theta0 = grass.get_inital_angle(slit_radius=self.params["slit_D"] / 2,
                                        wavelength=self.params["wavelength"],
                                        lens_curvature_radius=self.params["r_1"],
                                        grass_type="N-BK7")
        z_rel = grass.get_real_bfl(slit_radius=self.params["slit_D"] / 2,
                                   lens_curvature_radius=self.params["r_1"],
                                   lens_ct=self.params["ct_1"],
                                   wavelength=self.params["wavelength"], grass_type="N-BK7")
        dz = z_rel - self.params["bfl_1"]
        return 1, float(dz), float(np.tan(theta0))


def lambertian_exits(n: int, seed: int = 0):
    """Seeded synthetic exit photons: positions N(0, 1 mm) in x and y,
    Lambertian directions through the top face (v_z < 0), weights U[0.5, 1]
    (float32, the layout of get_result())."""
    rng = np.random.default_rng(seed)
    p = np.zeros((3, n), np.float32)
    p[0], p[1] = rng.normal(0, 1.0, n), rng.normal(0, 1.0, n)
    cos_t = np.sqrt(rng.random(n))
    phi = 2 * np.pi * rng.random(n)
    sin_t = np.sqrt(1 - cos_t ** 2)
    v = np.stack([sin_t * np.cos(phi), sin_t * np.sin(phi), -cos_t]).astype(np.float32)
    return p, v, rng.uniform(0.5, 1.0, n).astype(np.float32)


def main(argv=None) -> int:
    """``python -m pymonteopt_b200.optics``: time the default OBD scan on
    synthetic exit photons and print one JSON line."""
    import argparse
    ap = argparse.ArgumentParser(description=main.__doc__.split("\n")[0])
    ap.add_argument("--photons", type=int, default=4_000_000)
    ap.add_argument("--reps", type=int, default=3)
    args = ap.parse_args(argv)
    p, v, w = lambertian_exits(args.photons)
    m = OBD(seed=1)
    m.set_monte_data(p=p, v=v, w=w, nPh=args.photons)
    step, _ = m.opticalAnalysisMeth()                         # warm-up
    dev = E.require_cuda(None)
    dp_, dv, dw = (torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in (p, v, w))
    z = torch.from_numpy(step.astype(np.float64)).to(dev)
    out = torch.zeros(step.size, dtype=torch.float64, device=dev)
    prm = m._struct(z, step.size, 0, 0.0, 0.0)
    best = float("inf")
    for _ in range(args.reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        check(load().pmo_run_obd(C.byref(prm), dp_.data_ptr(), dv.data_ptr(), dw.data_ptr(),
                                 args.photons, out.data_ptr(), E._stream_handle()), "pmo_run_obd")
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    print(json.dumps({"photons": args.photons, "z_steps": int(step.size), "seconds": best,
                      "photon_z_traces_per_s": args.photons * step.size / best}))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
