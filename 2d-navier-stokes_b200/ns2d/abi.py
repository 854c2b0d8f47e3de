"""ctypes mirror of include/ns2d.h (types and constants only; loads nothing).

The layouts here must match the C header field for field; tests check the
struct size against the value the library reports.
"""
import ctypes as C

NS2D_ABI_VERSION = 2

# ns2d_status
OK, ERR_INVALID, ERR_UNSUPPORTED, ERR_CUDA, ERR_NOMEM, ERR_BLOWUP, ERR_DT, ERR_ITERS, ERR_STATE, ERR_NO_DEVICE = range(10)
STATUS_NAMES = {
    OK: "NS2D_OK", ERR_INVALID: "NS2D_ERR_INVALID", ERR_UNSUPPORTED: "NS2D_ERR_UNSUPPORTED",
    ERR_CUDA: "NS2D_ERR_CUDA", ERR_NOMEM: "NS2D_ERR_NOMEM", ERR_BLOWUP: "NS2D_ERR_BLOWUP",
    ERR_DT: "NS2D_ERR_DT", ERR_ITERS: "NS2D_ERR_ITERS", ERR_STATE: "NS2D_ERR_STATE",
    ERR_NO_DEVICE: "NS2D_ERR_NO_DEVICE",
}

NAVIER, EULER = 0, 1
RK4CN, RK4, AB4, DP5 = 0, 1, 2, 3
DEALIAS_23, DEALIAS_HOU_LI = 0, 1
FORCING_NONE, FORCING_KOLM, FORCING_ZERO = 0, 1, 2
FP64, FP32 = 0, 1
MODEL_FULL, MODEL_PHASE_ONLY = 0, 1
MAX_VORT, MAX_VEL, MAX_VORT_FOUR = 0, 1, 2
OBJ_ENSTROPHY, OBJ_PALINSTROPHY = 0, 1

QUIRK_CONJ_STATE = 1 << 0
QUIRK_HYPER_LATCH = 1 << 1
QUIRK_RK4_LINEAR = 1 << 2
QUIRK_HOU_LI_INT = 1 << 3
QUIRK_CFL_INDEX = 1 << 4
QUIRK_ENST_DISS = 1 << 5
QUIRKS_REFERENCE = 0x3F


class Params(C.Structure):
    """struct ns2d_params."""
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32),
        ("system", C.c_int32), ("integrator", C.c_int32), ("dealias", C.c_int32),
        ("forcing", C.c_int32), ("force_k", C.c_int32), ("quirks", C.c_int32),
        ("force_scale", C.c_double), ("nu", C.c_double), ("hyper_visc_pow", C.c_double),
        ("ekmn_alpha", C.c_double), ("ekmn_drag_pow", C.c_double),
        ("hyper_visc_flag", C.c_int32), ("ekmn_drag_flag", C.c_int32),
        ("adapt_step_flag", C.c_int32), ("cfl_cond_flag", C.c_int32),
        ("cfl_const", C.c_double), ("dt", C.c_double),
        ("precision", C.c_int32), ("flux_diagnostics", C.c_int32),
        ("device", C.c_int32), ("dealias_edge", C.c_int32), ("model", C.c_int32),
    ]

    def copy(self):
        p = Params()
        C.pointer(p)[0] = self
        return p


class Measures(C.Structure):
    """struct ns2d_measures (ComputeSystemMeasurables scalars)."""
    _fields_ = [(n, C.c_double) for n in (
        "energy", "enstrophy", "palinstrophy", "forcing_input", "divergence",
        "energy_diss", "enstrophy_diss",
        "d_enrg_dt_sbst", "enrg_flux_sbst", "enrg_diss_sbst",
        "d_enst_dt_sbst", "enst_flux_sbst", "enst_diss_sbst")]

    def as_list(self):
        return [getattr(self, n) for n, _ in self._fields_]


MEASURE_NAMES = [n for n, _ in Measures._fields_]
SPECTRA_NAMES = ["enrg", "enst", "d_enst_dt", "enst_flux", "enst_diss", "d_enrg_dt", "enrg_flux", "enrg_diss"]


# Parameter files written before the last int32 of ns2d_params was named
# dealias_edge call it "reserved" (its value was always 0).
_RENAMED = {"reserved": "dealias_edge"}


def params_from_arrays(names, values):
    """ns2d_params from parallel arrays of field names and values (the golden
    fixtures' param_names / params)."""
    types = dict(Params._fields_)
    kw = {}
    for n, v in zip(names, values):
        n = _RENAMED.get(str(n), str(n))
        kw[n] = float(v) if types[n].__name__ == "c_double" else int(v)
    return default_params(**kw)


def default_params(**kw):
    """Defaults of the reference's GetCMLArgs (Solver/src/utils.c:51-90) with the
    stock compile switches; keyword arguments override fields."""
    p = Params()
    p.nx = p.ny = 64
    p.system = NAVIER
    p.integrator = RK4CN
    p.dealias = DEALIAS_23
    p.forcing = FORCING_NONE
    p.force_k = 0
    p.quirks = QUIRKS_REFERENCE
    p.force_scale = 1.0
    p.nu = 1e-4
    p.hyper_visc_pow = 2.0
    p.ekmn_alpha = 0.0
    p.ekmn_drag_pow = -2.0
    p.hyper_visc_flag = 0
    p.ekmn_drag_flag = 0
    p.adapt_step_flag = 0
    p.cfl_cond_flag = 1
    p.cfl_const = 0.9
    p.dt = 1e-4
    p.precision = FP64
    p.flux_diagnostics = 1
    p.device = 0
    p.dealias_edge = 0
    p.model = MODEL_FULL
    for k, v in kw.items():
        if not hasattr(p, k):
            raise AttributeError(f"ns2d_params has no field {k!r}")
        setattr(p, k, v)
    return p
