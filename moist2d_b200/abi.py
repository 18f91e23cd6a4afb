"""ctypes mirror of include/moist2d.h (structs and constants).

Shared by the library binding (moist2d_b200._lib) and the oracle binding used by the tests.
"""
import ctypes as C

MOIST_F32 = 0
MOIST_F64 = 1

MOIST_OK = 0
MOIST_ERR_NAN = 1
MOIST_ERR_ARG = 2
MOIST_ERR_CUDA = 3
MOIST_ERR_TIMEOUT = 4
MOIST_ERR_UNSUPPORTED = 5
MOIST_ERR_NOMEM = 6
MOIST_ERR_IO = 7

MOIST_FLAG_TRI_NATIVE = 1
MOIST_FLAG_TRACER_WAVEFRONT = 2
MOIST_FLAG_TRACER_STREAM = 4
MOIST_FLAG_TRACER_DATAFLOW = 8
MOIST_NDIAG = 10

MOIST_KGROUP_PHYSICS = 0
MOIST_KGROUP_PROLOGUE = 1
MOIST_KGROUP_SUBSTEP = 2
MOIST_KGROUP_TRACER = 3
MOIST_KGROUP_UPDATE = 4
MOIST_KGROUP_OTHER = 5
MOIST_NGROUPS = 6

MOIST_HELPER_F2H = 0
MOIST_HELPER_KOREN = 1
MOIST_HELPER_SAT_VP = 2
MOIST_HELPER_SAT_Q = 3
MOIST_HELPER_EXP = 4
MOIST_HELPER_POW = 5

# the seven prognostic fields of State (moist.jl:296-302), in the order of the adjoint's arrays
PROGNOSTIC = ("rho", "rho_u", "rho_w", "rho_theta", "rho_qv", "rho_qc", "rho_qr")

# field names in the order compute_step! checks them for NaN (moist.jl:1543-1577)
NAN_FIELDS = ("rho", "rho_u", "rho_w", "rho_theta", "rho_qv", "rho_qc", "rho_qr",
              "d_rho_u_phys", "d_rho_theta_phys", "d_rho_qv_phys", "d_rho_qc_phys",
              "d_rho_qr_phys")


class moist_params(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("nz", C.c_int32), ("halo", C.c_int32), ("ns", C.c_int32),
        ("lx", C.c_double), ("h", C.c_double), ("dx", C.c_double),
        ("zf", C.c_void_p), ("dz", C.c_void_p), ("z", C.c_void_p),
        ("dt", C.c_double),
        ("nu", C.c_double), ("kappa", C.c_double), ("gamma_d", C.c_double),
        ("beta_offcenter", C.c_double), ("zf_sponge", C.c_double),
        ("do_mp", C.c_int32), ("do_auto", C.c_int32), ("do_accr", C.c_int32),
        ("do_revap", C.c_int32), ("do_sed", C.c_int32), ("do_rd", C.c_int32),
        ("do_sf", C.c_int32),
        ("cd", C.c_double), ("ch", C.c_double), ("ce", C.c_double), ("uabs_min", C.c_double),
        ("temp_surf", C.c_double),
        ("k_abs_qv", C.c_double), ("k_abs_qc", C.c_double), ("k_abs_qr", C.c_double),
        ("surf_emissivity", C.c_double), ("tau_cooling", C.c_double),
        ("z_tropopause", C.c_double),
        ("grav", C.c_double), ("rd", C.c_double), ("rv", C.c_double), ("cpd", C.c_double),
        ("cpv", C.c_double), ("cpl", C.c_double), ("cvd", C.c_double), ("p0", C.c_double),
        ("lv", C.c_double), ("sigma", C.c_double), ("epsvap", C.c_double),
        ("k_auto", C.c_double), ("qc_threshold", C.c_double), ("k_accr", C.c_double),
        ("k_evap", C.c_double), ("a_term", C.c_double), ("b_term", C.c_double),
        ("t0", C.c_double), ("es0", C.c_double), ("a_sat", C.c_double), ("b_sat", C.c_double),
        ("eps", C.c_double),
    ]


STATE_FIELDS = ("rho", "rho_u", "rho_w", "rho_theta", "rho_qv", "rho_qc", "rho_qr",
                "prec", "mflux", "shflux", "lhflux", "theta_ref",
                "d_rho_theta_mp", "d_rho_qv_mp", "d_rho_qc_mp", "d_rho_qr_mp", "d_rho_qr_sed",
                "d_rho_u_sf", "d_rho_theta_sf", "d_rho_qv_sf", "d_rho_theta_rd")


class moist_state_host(C.Structure):
    _fields_ = [(f, C.c_void_p) for f in STATE_FIELDS]


class moist_adjoint_seed(C.Structure):
    _fields_ = [("prec_weight", C.c_void_p), ("state", C.c_void_p * 7)]


class moist_adjoint_grad(C.Structure):
    _fields_ = [("state", C.c_void_p * 7), ("prec", C.c_void_p), ("k_auto", C.c_double),
                ("qc_threshold", C.c_double), ("objective", C.c_double), ("forward_ms", C.c_double),
                ("reverse_ms", C.c_double)]


class moist_bubble(C.Structure):
    _fields_ = [("xc", C.c_double), ("zc", C.c_double), ("radius", C.c_double), ("amp", C.c_double)]


class moist_init_profile(C.Structure):
    _fields_ = [(f, C.c_double) for f in ("theta0", "bndlayer_depth", "z_tropopause", "dtheta_dz_trop",
                                          "dtheta_dz_stra", "theta_pert", "rel_hum_surf", "rel_hum_decay",
                                          "u0")]
