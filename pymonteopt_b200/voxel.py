"""pymopt voxel-model API on the B200 engine.

Drop-in for ``pymopt.voxel_gpu`` (pymopt/voxel_gpu/_classes.py): the public
classes :class:`VoxelPlateModel`, :class:`VoxelPlateExModel` and
:class:`VoxelTuringModel` take the same constructor keywords, params keys and
methods (``build``, ``start``, ``get_result``, ``getRdTtRate``,
``getRdTtValues``, ``get_model_params``, ``save_result``), and add on-device
results: ``get_fluence``, ``get_Rr``, ``get_Tr``, ``get_A`` and the energy
ledger.

What runs where: the volume is built on the host exactly as the reference
builds it; ``start`` uploads it once, draws the photon source on the device
(the reference builds nPh-sized source arrays on the host and copies them,
pymopt/voxel_gpu/_classes.py:148-254), runs the transport kernel and the
tallies, and reads back a few hundred numbers.  Exit photons are exported
only when ``keep_exits`` is on (default: nPh <= 1e7), because they cost 28
bytes per photon on both sides of the PCIe link.
"""
from __future__ import annotations

import bz2
import datetime
import gc
import json
import pickle
import time
from abc import ABCMeta, abstractmethod

import numpy as np

from . import _abi as A
from .problem import TransportProblem, center_add
from .utils import ToJsonEncoder, calTime, set_params

__all__ = ["VoxelPlateModel", "VoxelPlateExModel", "VoxelTuringModel", "VoxelArrayModel",
           "PlateModel", "PlateExModel", "TuringModel_Rectangular", "TuringModel_Cylinder",
           "TuringModel_RnC"]


# =============================================================================
# Volume models (host geometry builders)
# =============================================================================

def _host_volume(shape) -> np.ndarray:
    """An uninitialised int8 host array for a label volume.  With a GPU
    present it is page-locked memory from torch's caching host allocator:
    a rebuilt model of the same size gets an already mapped block back (its
    fill takes no page faults), and start() uploads it by direct DMA.  The
    allocation initialises CUDA in the process, which start() does anyway."""
    import torch
    if torch.cuda.is_available():
        return torch.empty(tuple(int(s) for s in shape), dtype=torch.int8,
                           pin_memory=True).numpy()
    return np.empty(shape, dtype=np.int8)


class VoxelModel:
    """Base of the geometry builders (pymopt/voxel_gpu/_classes.py:387-394)."""

    def build(self):
        pass

    def set_params(self):
        pass

    def getModelSize(self):
        print("Memory area size for voxel storage: %0.3f Mbyte" % (self.voxel_model.nbytes * 1e-6))


class PlateModel(VoxelModel):
    """Layered slab (pymopt/voxel_gpu/_classes.py:396-468)."""

    def __init__(self):
        self.model_name = "PlateModel"
        self.dtype_f = np.float32
        self.dtype = np.int8
        self.params = {
            "x_size": 40, "y_size": 40,
            "voxel_space": 0.1,
            "thickness": [1.3, 40],
            "n": [1.5, 1.4],
            "n_air": 1.,
            "ma": [1e-5, 0.02374],
            "ms": [1e-5, 0.02374],
            "g": [0.9, 0.9],
        }
        self.keys = list(self.params.keys())
        self._param_instantiating()
        self.voxel_model = np.zeros((3, 3, 3), dtype=self.dtype)
        self.verbose = True

    def _param_instantiating(self):
        f = self.dtype_f
        self.thickness = self.params["thickness"]
        self.n = np.array(list(self.params["n"]) + [self.params["n_air"]]).astype(f)
        self.ms = np.array(self.params["ms"]).astype(f)
        self.ma = np.array(self.params["ma"]).astype(f)
        self.g = np.array(self.params["g"]).astype(f)
        self.voxel_space = self.params["voxel_space"]
        self.x_size = np.int32(round(self.params["x_size"] / self.params["voxel_space"]))
        self.y_size = np.int32(round(self.params["y_size"] / self.params["voxel_space"]))
        self.z_size = np.int32(round(np.array(self.thickness).sum() / self.params["voxel_space"]))

    @property
    def xy_size(self):
        return [self.params["x_size"], self.params["y_size"]]

    def build(self):
        self._make_voxel_model()
        if self.verbose:
            self.getModelSize()

    def set_params(self, *initial_data, **kwargs):
        set_params(self.params, self.keys, *initial_data, **kwargs)
        self._param_instantiating()

    def _make_voxel_model(self):
        # every (x, y) column of the slab is the same: the layer labels along
        # z between two shell voxels.  Writing that column across the plane is
        # one contiguous pass over the volume; filling layer by layer
        # (pymopt/voxel_gpu/_classes.py:437-457) writes short runs per column
        # and takes about twice as long.  The bytes are the same, except that
        # z voxels no layer reaches (rounded thicknesses that fall short of
        # z_size) hold label 0 here and uninitialised memory there.
        nz = self.z_size + 2
        col = np.zeros(nz, dtype=self.dtype)
        val = 1
        for n_, i in enumerate(self.thickness):
            val_ = round(i / self.voxel_space)
            col[val:val_ + val] = np.int8(n_)
            val += val_
        self.end_point = np.int8(np.array(self.thickness).size)
        col[0] = self.end_point
        col[-1] = self.end_point
        vm = _host_volume((self.x_size + 2, self.y_size + 2, nz))
        # the broadcast copy runs on torch's CPU thread pool (numpy's is one
        # thread); same bytes
        import torch
        torch.from_numpy(vm).copy_(torch.from_numpy(col).expand(vm.shape))
        for face in (np.s_[0, :, :], np.s_[-1, :, :], np.s_[:, 0, :], np.s_[:, -1, :]):
            vm[face] = self.end_point
        self.voxel_model = vm

    def get_params(self):
        return {"th": self.thickness, "ms": self.ms, "ma": self.ma, "n": self.n, "g": self.g}


class PlateExModel(VoxelModel):
    """Glass-enclosed two-layer sample (pymopt/voxel_gpu/_classes.py:470-551)."""

    def __init__(self):
        self.model_name = "PlateExModel"
        self.dtype = "int8"
        self.dtype_f = "float32"
        self.grass_num = 0
        self.intra_num = 1
        self.end_point = 2
        self.params = {
            "x_size": 40, "y_size": 40,
            "voxel_space": 0.1,
            "thickness": [1.3, 40],
            "n": [1.5, 1.4],
            "n_air": 1.,
            "ma": [1e-5, 0.02374],
            "ms": [1e-5, 0.02374],
            "g": [0.9, 0.9],
        }
        self.keys = list(self.params.keys())
        self._param_instantiating()
        self.voxel_model = np.zeros((3, 3, 3), dtype=self.dtype)
        self.model_shape = (3, 3, 3)
        self.verbose = True

    def _param_instantiating(self):
        f = self.dtype_f
        self.thickness = self.params["thickness"]
        self.n = np.array(list(self.params["n"]) + [self.params["n_air"]]).astype(f)
        self.ms = np.array(self.params["ms"]).astype(f)
        self.ma = np.array(self.params["ma"]).astype(f)
        self.g = np.array(self.params["g"]).astype(f)
        self.voxel_space = self.params["voxel_space"]
        self.x_size = int(self.params["x_size"] / self.params["voxel_space"])
        self.y_size = int(self.params["y_size"] / self.params["voxel_space"])
        self.z_size = int(self.params["thickness"][1] / self.params["voxel_space"])

    @property
    def xy_size(self):
        return [self.params["x_size"], self.params["y_size"]]

    def build(self):
        self._make_voxel_model()
        if self.verbose:
            self.getModelSize()

    def set_params(self, *initial_data, **kwargs):
        set_params(self.params, self.keys, *initial_data, **kwargs)
        self._param_instantiating()

    def _make_voxel_model(self):
        # the sample first, then a glass shell of num_pix+1 voxels on x, y and z
        self.num_pix = int(self.params["thickness"][0] / self.params["voxel_space"])
        k = self.num_pix + 1
        inner = np.full((self.x_size, self.y_size, self.z_size), self.intra_num, dtype=np.int8)
        vm = np.full((self.x_size + 2 * k, self.y_size + 2 * k, self.z_size + 2 * k),
                     self.grass_num, dtype=np.int8)
        vm[k:k + self.x_size, k:k + self.y_size, k:k + self.z_size] = inner
        for face in (np.s_[0, :, :], np.s_[-1, :, :], np.s_[:, 0, :], np.s_[:, -1, :],
                     np.s_[:, :, 0], np.s_[:, :, -1]):
            vm[face] = self.end_point
        self.voxel_model = vm

    def get_second_layer_addz(self):
        return self.num_pix + 1

    def get_params(self):
        return {"th": self.thickness, "ms": self.ms, "ma": self.ma, "n": self.n, "g": self.g}


def _add_array(X, num_pix, val, dtype, y_axis=False):
    """Pad ``num_pix`` voxels of ``val`` on z and x (and y) faces
    (pymopt/voxel_gpu/_classes.py:625-640)."""
    pads = [(num_pix, num_pix), (num_pix if y_axis else 0, num_pix if y_axis else 0),
            (num_pix, num_pix)]
    return np.pad(np.asarray(X, dtype=dtype), pads, mode="constant", constant_values=val)


class TuringModel_Rectangular(VoxelModel):
    """Trabecular bone in a rectangular cortical/subcutis/dermis shell
    (pymopt/voxel_gpu/_classes.py:554-666).  The bone volume comes from
    ``VoxelTuringModel.set_model(u)``; DICOM input needs pydicom and is not
    supported here."""

    _names = ["_space", "_trabecular", "_cortical", "_subcutaneus", "_dermis"]

    def __init__(self):
        self._init_model("TuringModel_Rectangular", {
            "xz_size": 17.15, "voxel_space": 0.0245, "dicom_path": False, "bv_tv": 0.138,
            "th_cortical": 1., "th_subcutaneus": 2.6, "th_dermis": 1.4,
            "n_space": 1., "n_trabecular": 1.4, "n_cortical": 1.4, "n_subcutaneus": 1.4,
            "n_dermis": 1.4, "n_air": 1.,
            "ma_space": 1e-8, "ma_trabecular": 0.02374, "ma_cortical": 0.02374,
            "ma_subcutaneus": 0.011, "ma_dermis": 0.037,
            "ms_space": 1e-8, "ms_trabecular": 20.54, "ms_cortical": 17.67,
            "ms_subcutaneus": 20, "ms_dermis": 20,
            "g_space": 0.90, "g_trabecular": 0.90, "g_cortical": 0.90, "g_subcutaneus": 0.90,
            "g_dermis": .90,
        }, end_point=5)

    def _init_model(self, name, params, end_point, air_num=None):
        self.model_name = name
        self.dtype_f = np.float32
        self.dtype = np.int8
        self.ct_num = 2
        self.subc_num = 3
        self.skin_num = 4
        if air_num is not None:
            self.air_num = air_num
        self.end_point = end_point
        self.voxel_model = np.zeros((3, 3, 3), dtype=self.dtype)
        self.params = params
        self.keys = list(self.params.keys())
        self._make_model_params()
        self.voxel_space = self.params["voxel_space"]
        self.verbose = True

    def build(self, bone_model):
        self.voxel_model = np.asarray(bone_model)
        self.voxel_space = self.params["voxel_space"]
        self._make_voxel_model()
        if self.verbose:
            self.getModelSize()

    def set_params(self, *initial_data, **kwargs):
        set_params(self.params, self.keys, *initial_data, **kwargs)
        self._make_model_params()

    def _make_model_params(self):
        _n, _ma, _ms, _g = [], [], [], []
        for i in self._names:
            _n.append(self.params["n" + i])
            _ma.append(self.params["ma" + i])
            _ms.append(self.params["ms" + i])
            _g.append(self.params["g" + i])
        _n.append(self.params["n_air"])
        self.n = np.array(_n).astype(self.dtype_f)
        self.ma = np.array(_ma).astype(self.dtype_f)
        self.ms = np.array(_ms).astype(self.dtype_f)
        self.g = np.array(_g).astype(self.dtype_f)

    def get_params(self):
        return {"ms": self.ms, "ma": self.ma, "n": self.n, "g": self.g}

    def _check_dicom(self):
        if self.params["dicom_path"]:
            raise NotImplementedError("DICOM input needs pydicom, which this engine does not "
                                      "use; pass the bone volume with set_model(u)")

    def add_array(self, X, num_pix, val, dtype, y_axis=False):
        return _add_array(X, num_pix, val, dtype, y_axis)

    def _shell_thickness(self):
        return np.round(np.array([self.params["th_cortical"], self.params["th_subcutaneus"],
                                  self.params["th_dermis"]]) /
                        self.params["voxel_space"]).astype(int)

    @staticmethod
    def _trim(A, vm):
        x = 0
        for i in A[:, int(A.shape[2] / 2), int(A.shape[0] / 2)]:
            if i:
                break
            x += 1
        if x == 0:
            return A, vm
        return A[x:-x, :, x:-x], vm[x:-x, :, x:-x]

    def _make_voxel_model(self):
        self._check_dicom()
        A = np.zeros_like(self.voxel_model).astype(bool)
        list_num = [self.ct_num, self.subc_num, self.skin_num]
        num_s = self._shell_thickness()
        int_num = int(self.voxel_model.shape[0] / 2 -
                      round(self.params["xz_size"] / (self.params["voxel_space"] * 2))) + num_s[0]
        A[int_num:-int_num, :, int_num:-int_num] = 1
        A, vm = self._trim(A, np.asarray(self.voxel_model, np.int8))
        for i in range(3):
            vm = self.add_array(vm, num_s[i], list_num[i], np.int8)
        self.voxel_model = self.add_array(vm, 1, self.end_point, np.int8, y_axis=True)


class TuringModel_Cylinder(TuringModel_Rectangular):
    """Cylindrical bone with concentric shells (pymopt/voxel_gpu/_classes.py:669-753)."""

    _names = ["_space", "_trabecular", "_cortical", "_subcutaneus", "_dermis", "_air"]

    _PARAMS = {
        "r_bone": 9.14, "voxel_space": 0.0245, "dicom_path": False, "bv_tv": 0.138,
        "th_cortical": 1., "th_subcutaneus": 2.6, "th_dermis": 1.4,
        "n_space": 1., "n_trabecular": 1.4, "n_cortical": 1.4, "n_subcutaneus": 1.4,
        "n_dermis": 1.4, "n_air": 1.,
        "ma_space": 1e-8, "ma_trabecular": 0.02374, "ma_cortical": 0.02374,
        "ma_subcutaneus": 0.011, "ma_dermis": 0.037, "ma_air": 1e-5,
        "ms_space": 1e-8, "ms_trabecular": 20.54, "ms_cortical": 17.67,
        "ms_subcutaneus": 20, "ms_dermis": 20, "ms_air": 1e-5,
        "g_space": 0.90, "g_trabecular": 0.90, "g_cortical": 0.90, "g_subcutaneus": 0.90,
        "g_dermis": .90, "g_air": .90,
    }

    def __init__(self):
        self._init_model("TuringModel_Cylinder", dict(self._PARAMS), end_point=6, air_num=5)

    @staticmethod
    def round_index(X, num_r):
        """(x, z) indices within radius ``num_r`` of the x-z centre
        (pymopt/voxel_gpu/_classes.py:708-715)."""
        size_x = int(X.shape[0] / 2)
        size_z = int(X.shape[2] / 2)
        x_lab = np.tile(np.arange(X.shape[0]), (X.shape[2], 1)).T - size_x
        y_lab = np.tile(np.arange(X.shape[2]), (X.shape[0], 1)) - size_z
        r_ = np.sqrt(x_lab ** 2 + y_lab ** 2)
        return np.where(r_ < num_r)

    def _disk(self, shape, num_r):
        A = np.zeros(shape, bool)
        ind = self.round_index(A, num_r)
        A[ind[0], :, ind[1]] = True
        return A

    def _shells(self, A, vm, num_tr, num_s):
        list_num = [self.ct_num, self.subc_num, self.skin_num]
        for i in range(3):
            B = self.add_array(A, num_s[i], False, bool)
            vm = self.add_array(vm, num_s[i], self.air_num, np.int8)
            num_tr += num_s[i]
            A = self._disk(B.shape, num_tr)
            vm[A & ~B] = list_num[i]
        return self.add_array(vm, 1, self.end_point, np.int8, y_axis=True)

    def _make_voxel_model(self):
        self._check_dicom()
        vm = np.array(self.voxel_model, np.int8)
        num_s = self._shell_thickness()
        num_tr = round(self.params["r_bone"] / self.params["voxel_space"]) - num_s[0]
        A = self._disk(vm.shape, num_tr)
        vm[~A] = self.air_num
        A, vm = self._trim(A, vm)
        self.voxel_model = self._shells(A, vm, num_tr, num_s)


class TuringModel_RnC(TuringModel_Cylinder):
    """Rectangle-and-cylinder bone (pymopt/voxel_gpu/_classes.py:755-821)."""

    def __init__(self):
        params = {"r_bone": 9.14, "xz_size": 17.15,
                  **{k: v for k, v in self._PARAMS.items() if k != "r_bone"}}
        self._init_model("TuringModel_RnC", params, end_point=6, air_num=5)

    def _make_voxel_model(self):
        self._check_dicom()
        vm = np.array(self.voxel_model, np.int8)
        num_s = self._shell_thickness()
        A = np.zeros(vm.shape, bool)
        int_num = int(vm.shape[0] / 2 -
                      round(self.params["xz_size"] / (self.params["voxel_space"] * 2))) + num_s[0]
        A[int_num:-int_num, :, int_num:-int_num] = True
        num_tr = round(self.params["r_bone"] / self.params["voxel_space"]) - num_s[0]
        A = A & self._disk(vm.shape, num_tr)
        vm[~A] = self.air_num
        A, vm = self._trim(A, vm)
        self.voxel_model = self._shells(A, vm, num_tr, num_s)


class ArrayModel(VoxelModel):
    """A caller-supplied padded label volume with per-label tables (no
    reference class; the reference calls ``vmc_kernel`` directly for these)."""

    def __init__(self, labels, voxel_space, end_point, ma, ms, g, n, vox_ma=None, vox_ms=None):
        self.model_name = "ArrayModel"
        self.voxel_model = np.asarray(labels, np.uint8)
        self.voxel_space = float(voxel_space)
        self.end_point = int(end_point)
        self.ma = np.asarray(ma, np.float32)
        self.ms = np.asarray(ms, np.float32)
        self.g = np.asarray(g, np.float32)
        self.n = np.asarray(n, np.float32)
        self.vox_ma = None if vox_ma is None else np.asarray(vox_ma, np.float32)
        self.vox_ms = None if vox_ms is None else np.asarray(vox_ms, np.float32)
        self.params = {}
        self.keys = []
        self.verbose = False

    def build(self):
        pass

    def set_params(self, *initial_data, **kwargs):
        set_params(self.params, self.keys, *initial_data, **kwargs)

    def get_params(self):
        return {"ms": self.ms, "ma": self.ma, "n": self.n, "g": self.g}


# =============================================================================
# Monte Carlo driver
# =============================================================================

class BaseVoxelMonteCarlo(metaclass=ABCMeta):
    """Shared driver (pymopt/voxel_gpu/_classes.py:41-382).

    Extra keywords beyond the reference's:
    ``nr``, ``dr`` — on-device R(r)/T(r) bins (bins (i*dr, (i+1)*dr], mm);
    ``fluence`` — tally absorbed weight per voxel for :meth:`get_fluence`;
    ``n_ang`` — on-device angle-resolved exit bins for :meth:`get_Ra` /
    :meth:`get_Ta`; ``n_line``, ``line_dr``, ``line_y_range`` — on-device
    side-face line profile for :meth:`get_line_profile`;
    ``keep_exits`` — export per-photon exit states for :meth:`get_result`
    (None: on when nPh <= 1e7); ``precision`` — 'fp32' (product) or 'fp64';
    ``verbose`` — the reference's progress prints.
    """

    @abstractmethod
    def __init__(self, *, nPh, model, dtype_f=np.float32, dtype=np.int32,
                 beam_type="TEM00", w_beam=0, beam_angle=0, initial_refrect_by_angle=False,
                 first_layer_clear=False, threadnum=None, nr=100, dr=0.1, fluence=False,
                 n_ang=0, n_line=0, line_dr=0.1, line_y_range=5.0,
                 keep_exits=None, precision="fp32", verbose=True, device=None):
        def __check_list_name(name, name_list):
            if name not in name_list:
                raise ValueError("%s is not a permitted for factor. Please choose from %s."
                                 % (name, name_list))

        self.beam_type_list = ["TEM00", False]
        __check_list_name(beam_type, self.beam_type_list)
        self.beam_type = beam_type
        self.dtype = dtype
        self.dtype_f = dtype_f
        self.nPh = nPh
        self.w_beam = w_beam
        self.initial_refrect_by_angle = initial_refrect_by_angle
        self.beam_angle = beam_angle
        self.model = model
        self.first_layer_clear = first_layer_clear
        # threads per block as in the reference (pymopt/voxel_gpu/_classes.py:70-73);
        # None leaves the launch shape to the engine (its tuned default)
        if threadnum is not None and threadnum > 1024:
            raise Exception("There are too many threads. threadnum < 1024.")
        self.threadnum = None if threadnum is None else int(threadnum)
        self.nr = int(nr)
        self.dr = float(dr)
        self.n_ang = int(n_ang)
        self.n_line = int(n_line)
        self.line_dr = float(line_dr)
        self.line_y_range = float(line_y_range)
        self.fluence = bool(fluence)
        self.fluence_mode = "voxel" if fluence else False
        self.keep_exits = keep_exits
        if precision not in ("fp32", "fp64"):
            raise ValueError("precision must be 'fp32' or 'fp64'")
        self.precision = precision
        self.verbose = verbose
        self.device = device
        self._dprob = None
        self._dprob_key = None
        self._tallies = None
        self.Rdw = self.Ttw = None
        self._reset_results()

    # ---- source (pymopt/voxel_gpu/_classes.py:155-254) -----------------------
    def _get_center_add(self, length):
        return center_add(length)

    def _initial_add(self):
        vm = self.model.voxel_model
        add = [self._get_center_add(vm.shape[0]), self._get_center_add(vm.shape[1]), 1]
        if self.first_layer_clear:
            add[2] = self.model.get_second_layer_addz()
        return add

    def _source(self):
        """Device-side source parameters equal to the host arrays the
        reference builds in _generate_initial_coodinate."""
        n = np.asarray(self.model.n, np.float32)
        l = self.model.voxel_space
        v = [0.0, 0.0, 1.0]
        spec_prob, spec_v = 0.0, [0.0, 0.0, -1.0]
        n1, n2 = n[-1], n[0]
        angled = self.beam_angle != 0 and self.w_beam == 0
        if angled:
            ai = self.beam_angle
            at = np.arcsin(np.sin(ai) * n1 / n2)
            v = [float(np.sin(at)), 0.0, float(np.cos(at))]
        rsp = 0.0
        if n1 != n2:
            rsp = ((n1 - n2) / (n1 + n2)) ** 2
            if angled:
                ai = self.beam_angle
                at = np.arcsin(np.sin(ai) * n1 / n2)
                rsp = ((np.sin(ai - at) / np.sin(ai + at)) ** 2 +
                       (np.tan(ai - at) / np.tan(ai + at)) ** 2) / 2
            elif self.first_layer_clear:
                n3 = n[1]
                r2 = ((n3 - n2) / (n3 + n2)) ** 2
                rsp = rsp + r2 * (1 - rsp) ** 2 / (1 - rsp * r2)
        w0 = np.float32(1.0) - np.float32(rsp)
        if angled and self.initial_refrect_by_angle:
            ai = self.beam_angle
            at = np.arcsin(np.sin(ai) * n1 / n2)
            spec_prob = float(((np.sin(ai - at) / np.sin(ai + at)) ** 2 +
                               (np.tan(ai - at) / np.tan(ai + at)) ** 2) / 2)
            spec_v = [float(np.sin(ai)), 0.0, float(-np.cos(ai))]
            w0 = np.float32(1.0)
        return dict(src_add=tuple(self._initial_add()), src_p=(0.0, 0.0, -l / 2),
                    src_v=tuple(v), src_w0=float(w0),
                    beam_sigma=float(self.w_beam) / 2 if self.w_beam else 0.0,
                    source=A.PMO_SRC_GAUSSIAN if self.w_beam else A.PMO_SRC_PENCIL,
                    spec_prob=spec_prob, spec_v=tuple(spec_v))

    def gaussianBeam(self, w=0.54, seed=None):
        """Lateral TEM00 samples x, y ~ N(0, w/2) (the reference draws them with
        scipy and plots them, pymopt/voxel_gpu/_classes.py:267-287; here they
        are drawn on the device inside start(), this helper is for inspection)."""
        rng = np.random.default_rng(seed)
        return rng.normal(0, w / 2, self.nPh), rng.normal(0, w / 2, self.nPh)

    def transport_problem(self) -> TransportProblem:
        m = self.model
        vm = np.asarray(m.voxel_model)
        n = np.asarray(m.n, np.float32)
        end = int(m.end_point)
        # the reference's int8 labels reinterpreted as uint8 (the same bytes
        # as astype for every value) without copying the volume
        labels = vm.view(np.uint8) if vm.dtype == np.int8 else vm.astype(np.uint8)
        prob = TransportProblem(
            labels=labels, voxel_space=float(m.voxel_space), end_label=end,
            ma=m.ma, ms=m.ms, g=m.g, n=n,
            center=(self._get_center_add(vm.shape[0]), self._get_center_add(vm.shape[1])),
            vox_ma=getattr(m, "vox_ma", None), vox_ms=getattr(m, "vox_ms", None),
            **self._source())
        return prob

    # ---- run ---------------------------------------------------------------
    def _device_problem(self):
        """The resident volume of this model.  A rebuilt model, or changed
        optical tables, get a fresh upload with its box map.  Otherwise the
        labels are uploaded again, as the reference's start() does
        (pymopt/voxel_gpu/_classes.py:92-101), and compared with the resident
        copy on the device, so that an in-place edit of ``model.voxel_model``
        between two starts replaces the volume and rebuilds the box map."""
        import torch
        from . import engine as E
        prob = self.transport_problem()
        key = (id(self.model.voxel_model), prob.labels.shape, prob.ma.tobytes(),
               prob.ms.tobytes(), prob.g.tobytes(), prob.n.tobytes())
        if self._dprob is None or self._dprob_key != key:
            self._dprob = E.DeviceProblem(prob, self.device)
            self._dprob_key = key
            return self._dprob
        dp = self._dprob
        fresh = torch.from_numpy(prob.labels).to(dp.device)
        if not torch.equal(fresh, dp.labels):
            prob.validate(labels=False)
            E.check_labels(fresh, prob.end_label, prob.n_labels)
            dp.labels.copy_(fresh)
            if dp.words is not None:
                dp.build_words()
        dp.host = prob  # the source may have changed too (beam settings)
        return dp

    def start(self, rand_seed=None):
        from . import engine as E
        if rand_seed is None:
            rand_seed = np.random.randint(1e5)
        self.nPh = int(self.nPh)
        self._reset_results()
        dp = self._device_problem()
        keep = self.keep_exits if self.keep_exits is not None else self.nPh <= 10_000_000
        spec = E.TallySpec(nr=self.nr, dr=self.dr,
                           fluence=A.PMO_FLU_GLOBAL if self.fluence else A.PMO_FLU_NONE,
                           export_exits=bool(keep), n_ang=self.n_ang, n_line=self.n_line,
                           line_dr=self.line_dr, line_y_range=self.line_y_range)
        if self.verbose:
            print("")
            print("###### Start (Random seed: %s) ######" % rand_seed)
            print("")
        start_ = time.time()
        tal = E.Tallies(dp, spec, self.nPh)
        bt = 0 if self.threadnum is None else max(32, min(512, 32 * round(self.threadnum / 32)))
        E.run_plain(dp, self.nPh, int(rand_seed), tallies=tal,
                    precision=A.PMO_FP64 if self.precision == "fp64" else A.PMO_FP32,
                    block_threads=bt)
        tal.check()  # synchronises; raises on device-side errors
        self._tallies = tal
        self.rand_seed = rand_seed
        self._end_process(keep)
        if self.verbose:
            print("###### End ######")
        self.getRdTtRate()
        if self.verbose:
            calTime(time.time(), start_)
        return self

    def _end_process(self, keep):
        tal = self._tallies
        self._ledger = tal.ledger.cpu().numpy()
        self._counters = tal.host_counters()
        if keep:
            self.add_result = tal.exit_add.cpu().numpy().astype(self.dtype)
            self.p_result = tal.exit_p.cpu().numpy().astype(self.dtype_f)
            self.v_result = tal.exit_v.cpu().numpy().astype(self.dtype_f)
            self.w_result = tal.exit_w.cpu().numpy().astype(self.dtype_f)
        else:
            self._reset_results()

    def _reset_results(self):
        self.v_result = np.empty((3, 0)).astype(self.dtype_f)
        self.p_result = np.empty((3, 0)).astype(self.dtype_f)
        self.add_result = np.empty((3, 0)).astype(self.dtype)
        self.w_result = np.empty(0).astype(self.dtype_f)
        return self

    def get_voxel_model(self):
        return self.model.voxel_model

    # ---- results -----------------------------------------------------------
    def _encooder(self, p, add):
        """Exit position in model coordinates (pymopt/voxel_gpu/_classes.py:302-310)."""
        space = self.model.voxel_space
        cx = self._get_center_add(self.model.voxel_model.shape[0])
        cy = self._get_center_add(self.model.voxel_model.shape[1])
        enc = p.copy()
        enc[0] = space * (add[0] - cx) + p[0]
        enc[1] = space * (add[1] - cy) + p[1]
        enc[2] = np.round(space * (add[2] - 1) + p[2] + space / 2, 6)
        return enc

    def get_result(self):
        if self._tallies is not None and self.w_result.size == 0 and self.nPh > 0:
            raise RuntimeError("exit photons were not exported (keep_exits=False); "
                               "use get_Rr / get_Tr / getRdTtValues for the on-device tallies")
        return {"p": self._encooder(self.p_result, self.add_result), "v": self.v_result,
                "w": self.w_result, "nPh": self.nPh}

    def get_model_params(self):
        return self.model.get_params()

    def set_monte_params(self, *, nPh, model, dtype_f=np.float32, dtype=np.int32, w_beam=0):
        self.dtype = dtype
        self.dtype_f = dtype_f
        self.nPh = nPh
        self.w_beam = w_beam
        self.model = model

    def build(self, *initial_data, **kwargs):
        if initial_data == () and kwargs == {}:
            pass
        else:
            self.model.set_params(*initial_data, **kwargs)
        self.model.verbose = self.verbose
        self.model.build()

    def getRdTtRate(self):
        """Rd / Tt as the reference defines them: exit weight with v_z < 0 /
        v_z > 0 over nPh (pymopt/voxel_gpu/_classes.py:326-334)."""
        L = self._ledger
        self.Rdw = float(L[A.PMO_L_RD] / self.nPh)
        self.Ttw = float(L[A.PMO_L_TT] / self.nPh)
        if self.verbose:
            print("######")
            print("Mean Rd %0.6f" % self.Rdw)
            print("Mean Td %0.6f" % self.Ttw)
            print()

    def getRdTtValues(self):
        return {"Rd": self.Rdw, "Td": self.Ttw, "Tt": self.Ttw, "A": self.get_A()}

    def get_A(self):
        """Absorbed fraction (FP64 ledger of implicit-capture deposits)."""
        return float(self._ledger[A.PMO_L_ABS] / self.nPh)

    def get_ledger(self) -> dict:
        """Energy ledger per launched photon (all FP64 sums / nPh)."""
        L = self._ledger / self.nPh
        names = {"w_init": A.PMO_L_WINIT, "Rd": A.PMO_L_RD, "Tt": A.PMO_L_TT,
                 "exit_vz0": A.PMO_L_EXIT0, "A": A.PMO_L_ABS, "roulette_gain": A.PMO_L_RGAIN,
                 "roulette_loss": A.PMO_L_RLOSS, "error_weight": A.PMO_L_ERRW,
                 "Rd_top": A.PMO_L_RD_TOP, "Tt_bottom": A.PMO_L_TT_BOTTOM,
                 "specular": A.PMO_L_SPEC}
        out = {k: float(L[i]) for k, i in names.items()}
        out["balance"] = (out["w_init"] + out["roulette_gain"] - out["Rd"] + out["specular"]
                          - out["Tt"] - out["exit_vz0"] - out["A"] - out["roulette_loss"]
                          - out["error_weight"])
        return out

    def get_counters(self) -> dict:
        c = self._counters
        return {"photons": int(c[A.PMO_C_PHOTONS]), "interactions": int(c[A.PMO_C_INTERACT]),
                "crossings": int(c[A.PMO_C_CROSS]), "fresnel": int(c[A.PMO_C_FRESNEL]),
                "reflections": int(c[A.PMO_C_REFLECT]), "roulette": int(c[A.PMO_C_ROULETTE]),
                "exits": int(c[A.PMO_C_EXITS])}

    def _profile(self, cats, surface_only):
        rr = self._tallies.rr.cpu().numpy().astype(np.float64)
        prof = rr[cats[0]] + (0 if surface_only else rr[cats[1]])
        da = np.array([2 * np.pi * (i + 0.5) * self.dr ** 2 for i in range(self.nr)])
        alpha = np.array([i * self.dr for i in range(self.nr)])
        return alpha, prof / (da * self.nPh)

    def get_Rr(self, surface_only=False):
        """R(r) [mm^-2] of exits with v_z < 0 (``surface_only``: through the
        top face only), binned like metrics.radialDistance."""
        return self._profile((A.PMO_RR_TOP, A.PMO_RR_LAT_NEG), surface_only)

    def get_Tr(self, surface_only=False):
        return self._profile((A.PMO_RR_BOTTOM, A.PMO_RR_LAT_POS), surface_only)

    def _angular(self, row):
        if self._tallies is None or self._tallies.ang is None:
            raise RuntimeError("construct the model with n_ang > 0 for angle-resolved exits")
        nn = self.n_ang
        da = np.pi / (2 * nn)
        alpha = np.array([(i + 0.5) * da for i in range(nn + 1)])
        do = 4 * np.pi * np.sin(alpha) * np.sin(da / 2)
        h = self._tallies.ang[row].cpu().numpy().astype(np.float64)
        return alpha[:-1], h / (do[:-1] * self.nPh)

    def get_Ra(self):
        """Angle-resolved reflectance of exits with v_z < 0 [sr^-1], as
        metrics.angularyResolved on them (pymopt/metrics/_scoring.py:27-38)."""
        return self._angular(0)

    def get_Ta(self):
        """Angle-resolved transmittance of exits with v_z > 0 [sr^-1]."""
        return self._angular(1)

    def get_line_profile(self):
        """Depth profile [mm^-2] of exits moving towards -x within
        |y| < line_y_range, as metrics.lineDistance on them
        (pymopt/metrics/_scoring.py:40-51; pymopt/virtualOBD.py:171-172)."""
        if self._tallies is None or self._tallies.line is None:
            raise RuntimeError("construct the model with n_line > 0 for the line profile")
        nn, dr = self.n_line, self.line_dr
        alpha = np.array([i * dr for i in range(nn + 1)])
        da = np.ones(nn) * dr * self.line_y_range * 2
        h = self._tallies.line.cpu().numpy().astype(np.float64)
        return alpha[:-1], h / (da * self.nPh)

    def get_fluence(self):
        """Fluence per voxel of the interior (shell stripped), FP64:
        phi = absorbed weight / (nPh * l^3 * mu_a) [mm^-2]."""
        from . import engine as E
        if not self.fluence:
            raise RuntimeError("construct the model with fluence=True to tally fluence")
        return E.normalize_fluence(self._dprob, self._tallies).cpu().numpy()

    def get_absorbed(self):
        """Absorbed weight per voxel of the padded grid, divided by nPh."""
        from . import engine as E
        return E.absorbed_weight(self._tallies).cpu().numpy() / self.nPh

    # ---- persistence (pymopt/voxel_gpu/_classes.py:338-382) -----------------
    def save_result(self, fname, *, coment="", save_monte=True, save_params=True):
        start_ = time.time()
        if save_monte:
            res = self.get_result()
            save_name = fname + "_LID.pkl.bz2"
            with bz2.open(save_name, "wb") as fp:
                fp.write(pickle.dumps(res))
            if self.verbose:
                print("Monte Carlo results saved in ")
                print("-> %s" % save_name)
                print("")
        if save_params:
            info = self._calc_info(coment)
            save_name = fname + "_info.json"
            with open(save_name, "w") as fp:
                json.dump(info, fp, indent=4, cls=ToJsonEncoder)
            if self.verbose:
                print("Calculation conditions are saved in")
                print("-> %s" % save_name)
                print("")
        if self.verbose:
            calTime(time.time(), start_)

    def _calc_info(self, coment=""):
        _params = self.model.get_params()
        return {
            "Date": datetime.datetime.now().isoformat(),
            "coment": coment,
            "number_of_photons": self.nPh,
            "calc_dtype": "32 bit" if self.precision == "fp32" else "64 bit",
            "model": {
                "model_name": self.model.model_name,
                "model_params": _params,
                "model_voxel_space": self.model.voxel_space,
                "model_xy_size": getattr(self.model, "xy_size", None),
            },
            "w_beam": self.w_beam,
            "beam_angle": self.beam_angle,
            "initial_refrect_mode": self.initial_refrect_by_angle,
            "beam_mode": "TEM00",
            "fluence_mode": self.fluence_mode,
        }

    def release(self):
        """Free the device copies of the volume and the tallies."""
        self._dprob = None
        self._tallies = None
        gc.collect()


class VoxelPlateModel(BaseVoxelMonteCarlo):
    def __init__(self, *, nPh=1000, dtype_f=np.float32, dtype=np.int32, beam_type="TEM00",
                 w_beam=0, beam_angle=0, initial_refrect_by_angle=False, first_layer_clear=False,
                 threadnum=None, **kw):
        super().__init__(nPh=nPh, model=PlateModel(), dtype_f=dtype_f, dtype=dtype,
                         w_beam=w_beam, beam_angle=beam_angle, beam_type=beam_type,
                         initial_refrect_by_angle=initial_refrect_by_angle,
                         first_layer_clear=first_layer_clear, threadnum=threadnum, **kw)


class VoxelPlateExModel(BaseVoxelMonteCarlo):
    def __init__(self, *, nPh=1000, dtype_f=np.float32, dtype=np.int32, beam_type="TEM00",
                 w_beam=0, beam_angle=0, initial_refrect_by_angle=False, first_layer_clear=True,
                 threadnum=None, **kw):
        super().__init__(nPh=nPh, model=PlateExModel(), dtype_f=dtype_f, dtype=dtype,
                         w_beam=w_beam, beam_angle=beam_angle, beam_type=beam_type,
                         initial_refrect_by_angle=initial_refrect_by_angle,
                         first_layer_clear=first_layer_clear, threadnum=threadnum, **kw)

    def set_params(self, *initial_data, **kwargs):
        self.model.set_params(*initial_data, **kwargs)

    def _calc_info(self, coment=""):
        info = super()._calc_info(coment)
        info["model"] = {"model_name": self.model.model_name, "model_params": self.model.params}
        info.pop("fluence_mode", None)
        return info


class VoxelTuringModel(BaseVoxelMonteCarlo):
    def __init__(self, *, nPh=1000, dtype_f=np.float32, dtype=np.int32, beam_type="TEM00",
                 w_beam=0, beam_angle=0, initial_refrect_by_angle=False, first_layer_clear=False,
                 threadnum=None, model_name="TuringModel", **kw):
        self.namelist = ["TuringModel_Rectangular", "TuringModel_Cylinder", "TuringModel_RnC"]
        if model_name == self.namelist[0]:
            model = TuringModel_Rectangular()
        elif model_name == self.namelist[1]:
            model = TuringModel_Cylinder()
        elif model_name == self.namelist[2]:
            model = TuringModel_RnC()
        else:
            # the reference prints and then fails on the unbound name
            raise ValueError("Invalid name: %s (choose from %s)" % (model_name, self.namelist))
        super().__init__(nPh=nPh, model=model, dtype_f=dtype_f, dtype=dtype, w_beam=w_beam,
                         beam_angle=beam_angle, beam_type=beam_type,
                         initial_refrect_by_angle=initial_refrect_by_angle,
                         first_layer_clear=first_layer_clear, threadnum=threadnum, **kw)
        self.bone_model = False

    def _initial_add(self):
        add = super()._initial_add()
        if self.model.model_name == self.namelist[1]:
            # first z where the column holds the skin label (end_point - 2)
            col = self.model.voxel_model[add[0], add[1]]
            hits = np.flatnonzero(col == self.model.end_point - 2)
            if hits.size == 0:
                raise ValueError("no skin voxel on the beam axis")
            add[2] = int(hits[0])
        return add

    def build(self, *initial_data, **kwargs):
        if not (initial_data == () and kwargs == {}):
            self.model.set_params(*initial_data, **kwargs)
        self.model.verbose = self.verbose
        self.model.build(self.bone_model)
        del self.bone_model

    def set_model(self, u):
        self.bone_model = u

    def set_params(self, *initial_data, **kwargs):
        self.model.set_params(*initial_data, **kwargs)

    def _calc_info(self, coment=""):
        info = super()._calc_info(coment)
        info["model"] = {"model_name": self.model.model_name, "model_params": self.model.params}
        info.pop("fluence_mode", None)
        return info


class VoxelArrayModel(BaseVoxelMonteCarlo):
    """Transport in a caller-supplied padded label volume (C3-style
    heterogeneous media; per-voxel ma/ms with ``vox_ma``/``vox_ms``)."""

    def __init__(self, labels, voxel_space, end_point, ma, ms, g, n, *, nPh=1000,
                 vox_ma=None, vox_ms=None, **kw):
        super().__init__(nPh=nPh, model=ArrayModel(labels, voxel_space, end_point, ma, ms, g, n,
                                                   vox_ma, vox_ms), **kw)

    def _initial_add(self):
        vm = self.model.voxel_model
        return [self._get_center_add(vm.shape[0]), self._get_center_add(vm.shape[1]), 1]

    def _source(self):
        src = super()._source()
        # n[0] of the reference is the first layer; here the label under the beam
        n = np.asarray(self.model.n, np.float32)
        ix, iy, iz = src["src_add"]
        n1, n2 = n[self.model.end_point], n[int(self.model.voxel_model[ix, iy, iz])]
        rsp = ((n1 - n2) / (n1 + n2)) ** 2 if n1 != n2 else np.float32(0)
        src["src_w0"] = float(np.float32(1.0) - np.float32(rsp))
        return src
