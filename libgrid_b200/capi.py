"""ctypes view of the libgrid C ABI (structs and prototypes).

The same declarations describe two libraries:
  * libgrid_b200.so, whose structs follow the reference's USE_CUDA layout
    (src/structs.h:24-103 with the cuFFT handle and host-lock fields), and
  * a CPU-only build of the reference itself (same structs without those
    fields), used by the tests as the oracle.
Complex arguments and results (C `double _Complex`) are passed as a struct of
two doubles, which the x86-64 System V ABI classifies identically.
"""
from __future__ import annotations

import ctypes as C

c_double_p = C.POINTER(C.c_double)


class Complex(C.Structure):
    _fields_ = [("re", C.c_double), ("im", C.c_double)]

    @classmethod
    def of(cls, z) -> "Complex":
        z = complex(z)
        return cls(z.real, z.imag)

    def value(self) -> complex:
        return complex(self.re, self.im)


def _make_structs(cuda_layout: bool):
    class CGrid(C.Structure):
        pass

    CBC = C.CFUNCTYPE(Complex, C.POINTER(CGrid), C.c_long, C.c_long, C.c_long)
    fields = [
        ("value", C.c_void_p),
        ("id", C.c_char * 32),
        ("grid_len", C.c_size_t),
        ("nx", C.c_long),
        ("ny", C.c_long),
        ("nz", C.c_long),
        ("step", C.c_double),
        ("x0", C.c_double),
        ("y0", C.c_double),
        ("z0", C.c_double),
        ("kx0", C.c_double),
        ("ky0", C.c_double),
        ("kz0", C.c_double),
        ("omega", C.c_double),
        ("value_outside", C.c_void_p),
        ("outside_params_ptr", C.c_void_p),
        ("default_outside_params", C.c_double * 2),
        ("plan", C.c_void_p),
        ("iplan", C.c_void_p),
    ]
    if cuda_layout:
        fields += [("cufft_handle", C.c_int), ("host_lock", C.c_char)]
    fields += [("fft_norm", C.c_double), ("fft_norm2", C.c_double), ("flag", C.c_char)]
    CGrid._fields_ = fields

    class RGrid(C.Structure):
        pass

    rfields = [
        ("value", C.c_void_p),
        ("id", C.c_char * 32),
        ("grid_len", C.c_size_t),
        ("nx", C.c_long),
        ("ny", C.c_long),
        ("nz", C.c_long),
        ("nz2", C.c_long),
        ("step", C.c_double),
        ("x0", C.c_double),
        ("y0", C.c_double),
        ("z0", C.c_double),
        ("kx0", C.c_double),
        ("ky0", C.c_double),
        ("kz0", C.c_double),
        ("value_outside", C.c_void_p),
        ("outside_params_ptr", C.c_void_p),
        ("default_outside_params", C.c_double),
        ("plan", C.c_void_p),
        ("iplan", C.c_void_p),
    ]
    if cuda_layout:
        rfields += [("cufft_handle_r2c", C.c_int), ("cufft_handle_c2r", C.c_int), ("host_lock", C.c_char)]
    rfields += [("fft_norm", C.c_double), ("fft_norm2", C.c_double), ("flag", C.c_char)]
    RGrid._fields_ = rfields

    class WF(C.Structure):
        _fields_ = [
            ("grid", C.POINTER(CGrid)),
            ("mass", C.c_double),
            ("norm", C.c_double),
            ("cfft_width", C.c_double),
            ("boundary", C.c_char),
            ("propagator", C.c_char),
            ("cworkspace", C.POINTER(CGrid)),
            ("cworkspace2", C.POINTER(CGrid)),
            ("cworkspace3", C.POINTER(CGrid)),
            ("ts_func", C.c_void_p),
            ("lx", C.c_long),
            ("hx", C.c_long),
            ("ly", C.c_long),
            ("hy", C.c_long),
            ("lz", C.c_long),
            ("hz", C.c_long),
            ("kmax", C.c_double),
        ]

    return CGrid, RGrid, WF, CBC


# Constants of the reference's src/defs.h:20-32.
WF_DIRICHLET_BOUNDARY = 1
WF_NEUMANN_BOUNDARY = 2
WF_PERIODIC_BOUNDARY = 3
WF_2ND_ORDER_FFT = 1
WF_4TH_ORDER_FFT = 2
WF_2ND_ORDER_CFFT = 3
WF_4TH_ORDER_CFFT = 4
WF_2ND_ORDER_CN = 5
WF_4TH_ORDER_CN = 6
WF_1ST_ORDER_EULER = 7
GRID_PREC_FP64 = 0
GRID_PREC_FP32 = 1
GRID_AUTOAMU = 1.0 / 1822.88853006


def bind(lib: C.CDLL, cuda_layout: bool, extensions: bool):
    """Attach argtypes/restypes for the libgrid API to `lib`; return structs."""
    CGrid, RGrid, WF, CBC = _make_structs(cuda_layout)
    PC, PR, PW = C.POINTER(CGrid), C.POINTER(RGrid), C.POINTER(WF)
    L, D, V, Cx, ch = C.c_long, C.c_double, C.c_void_p, Complex, C.c_char

    def f(name, res, *args):
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = list(args)

    f("grid_threads_init", None, L)
    f("grid_wf_analyze_method", None, ch)
    f("cgrid_alloc", PC, L, L, L, D, V, V, C.c_char_p)
    f("cgrid_free", None, PC)
    f("cgrid_copy", None, PC, PC)
    f("cgrid_zero", None, PC)
    f("cgrid_constant", None, PC, Cx)
    f("cgrid_set_momentum", None, PC, D, D, D)
    f("cgrid_set_origin", None, PC, D, D, D)
    f("cgrid_set_rotation", None, PC, D)
    f("grid_random_seed", None, L, L, L, L)
    f("rgrid_random_uniform", None, PR, D)
    f("rgrid_random_normal", None, PR, D)
    f("cgrid_random_uniform", None, PC, Cx)
    f("cgrid_random_uniform_sp", None, PC, D)
    f("cgrid_random_normal", None, PC, Cx)
    f("cgrid_random_normal_sp", None, PC, D)
    f("cgrid_fft", None, PC)
    f("cgrid_inverse_fft", None, PC)
    f("cgrid_inverse_fft_norm", None, PC)
    f("cgrid_inverse_fft_norm2", None, PC)
    f("cgrid_multiply", None, PC, Cx)
    f("cgrid_sum", None, PC, PC, PC)
    f("cgrid_difference", None, PC, PC, PC)
    f("cgrid_product", None, PC, PC, PC)
    f("cgrid_conjugate_product", None, PC, PC, PC)
    f("cgrid_add_scaled", None, PC, Cx, PC)
    f("cgrid_add_scaled_product", None, PC, Cx, PC, PC)
    f("cgrid_integral", Cx, PC)
    f("cgrid_integral_of_square", D, PC)
    f("cgrid_integral_of_conjugate_product", Cx, PC, PC)
    f("cgrid_grid_expectation_value", Cx, PC, PC)
    f("cgrid_value_at_index", Cx, PC, L, L, L)
    f("cgrid_value_to_index", None, PC, L, L, L, Cx)
    f("cgrid_fd_laplace", None, PC, PC)
    f("cgrid_fd_laplace_x", None, PC, PC)
    f("cgrid_fd_laplace_y", None, PC, PC)
    f("cgrid_fd_laplace_z", None, PC, PC)
    f("cgrid_fd_gradient_x", None, PC, PC)
    f("cgrid_fd_gradient_y", None, PC, PC)
    f("cgrid_fd_gradient_z", None, PC, PC)
    f("cgrid_fft_laplace", None, PC, PC)
    f("cgrid_fft_gradient_x", None, PC, PC)
    f("cgrid_fft_gradient_y", None, PC, PC)
    f("cgrid_fft_gradient_z", None, PC, PC)
    f("cgrid_fft_laplace_expectation_value", D, PC)
    f("cgrid_add", None, PC, Cx)
    f("cgrid_fft_convolute", None, PC, PC, PC)
    f("cgrid_extrapolate", None, PC, PC)
    f("cgrid_write", None, PC, V)
    f("cgrid_read", PC, PC, V)
    f("rgrid_alloc", PR, L, L, L, D, V, V, C.c_char_p)
    f("rgrid_free", None, PR)
    f("rgrid_fd_laplace", None, PR, PR)
    f("rgrid_fft", None, PR)
    f("rgrid_inverse_fft_norm", None, PR)
    f("rgrid_inverse_fft", None, PR)
    f("rgrid_inverse_fft_norm2", None, PR)
    f("rgrid_integral", D, PR)
    f("rgrid_sum", None, PR, PR, PR)
    f("rgrid_product", None, PR, PR, PR)
    f("rgrid_multiply", None, PR, D)
    f("rgrid_fft_convolute", None, PR, PR, PR)
    f("rgrid_extrapolate", None, PR, PR)
    f("rgrid_write", None, PR, V)
    f("rgrid_read", PR, PR, V)
    f("grid_real_to_complex_re", None, PC, PR)
    f("grid_product_norm", None, PR, PR, PC)
    f("grid_product_complex_with_real", None, PC, PR)
    f("grid_grid_expectation_value", D, PC, PR)
    f("grid_wf_alloc", PW, L, L, L, D, D, ch, ch, C.c_char_p)
    f("grid_wf_free", None, PW)
    f("grid_wf_boundary", None, PW, PW, L, L, L, L, L, L)
    f("grid_wf_propagate", None, PW, PC, Cx)
    f("grid_wf_propagate_potential", None, PW, Cx, PC, D)
    f("grid_wf_propagate_kinetic_fft", None, PW, Cx)
    f("grid_wf_propagate_kinetic_cfft", None, PW, Cx)
    f("grid_wf_propagate_kinetic_cn", None, PW, Cx)
    f("grid_wf_propagate_predict", None, PW, PW, PC, Cx)
    f("grid_wf_propagate_correct", None, PW, PC, Cx)
    f("grid_wf_norm", D, PW)
    f("grid_wf_normalize", D, PW)
    f("grid_wf_energy", D, PW, PR)
    f("grid_wf_kinetic_energy", D, PW)
    f("grid_wf_potential_energy", D, PW, PR)
    f("grid_wf_energy_fft", D, PW, PR)
    f("grid_wf_energy_cn", D, PW, PR)
    f("grid_wf_kinetic_energy_fft", D, PW)
    f("grid_wf_kinetic_energy_cn", D, PW)
    f("grid_wf_density", None, PW, PR)
    f("grid_wf_overlap", Cx, PW, PW)
    f("grid_wf_energy_and_error", D, PW, PC, PC, C.POINTER(D))
    if cuda_layout:
        f("cuda_enable", None, ch, C.c_int, C.POINTER(C.c_int))
        f("cuda_status", ch)
        f("cuda_remove_block", C.c_int, V, ch)
    if extensions:
        f("grid_wf_propagate_gp", None, PW, PR, D, Cx)
        f("grid_wf_propagate_n", None, PW, PC, Cx, L)
        f("grid_wf_propagate_gp_n", None, PW, PR, D, Cx, L)
        f("grid_wf_precision", None, PW, ch)
        f("grid_wf_get_precision", ch, PW)
        f("grid_wf_batch_alloc", V, C.POINTER(PW), C.POINTER(PC), L, Cx)
        f("grid_wf_batch_propagate", None, V, L)
        f("grid_wf_batch_free", None, V)
        f("grid_wf_batch_threads", C.c_int, V)
        f("gb_grid_sync_host", None, V)
        f("gb_grid_host_modified", None, V)
        f("gb_last_error", C.c_int)
        f("gb_synchronize", C.c_int)
        f("gb_clear_error", None)
        f("gb_last_error_where", C.c_char_p)
        f("gb_wait_limit", C.c_uint, C.c_uint)
        f("gb_chain_lag", C.c_int, C.c_int)
        f("gb_cn_warp_solver", C.c_int, C.c_int)
        f("gb_pass_error_flag", C.c_int, C.c_int)
        f("gb_cn_error_flag", C.c_int)
        f("gb_batch_error_flag", C.c_int, V, C.c_int)
        f("gb_launch_count", L)
        f("gb_event_record", C.c_int, C.c_int)
        f("gb_event_elapsed_ms", C.c_float, C.c_int, C.c_int)
    return CGrid, RGrid, WF, CBC
