"""Python mirror of the ccmm-rs evaluation interface over libckks_b200.so.

The compute path is the sm_100a CUDA library behind the C ABI in
include/ckks_b200.h; this module only marshals torch CUDA tensors (device
memory) and host numpy arrays into those calls. There is no CPU fallback: if
the library or a GPU is missing, calls raise.

Names follow the reference crate (ring/, ckks/, grafting/):
  RnsNttPlan / PreparedRnsNttPlan    ring/rns_ntt.rs, ring/prepared_rns_ntt.rs
  rotate / rotate_hoisted            ckks/hybrid_rns_galois_key.rs
  tensor / relinearize               grafting/rns_key_switch.rs, grafting/bounded_key_switch.rs
  multiply_relinearize_rescale       ckks/rns_multiply.rs
  multiply_plain                     ckks/rns_plain_multiply.rs
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(PKG)
LIB_PATH = os.path.join(PKG, "_build", "libckks_b200.so")
HEADER = os.path.join(ROOT, "include", "ckks_b200.h")

U32, U64, I32, VP = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int32, ctypes.c_void_p
u64p = ctypes.POINTER(ctypes.c_uint64)
u32p = ctypes.POINTER(ctypes.c_uint32)
i8p = ctypes.POINTER(ctypes.c_int8)

_SIGS = {
    "ckks_last_error_string": (ctypes.c_char_p, []),
    "ckks_version": (ctypes.c_char_p, []),
    "ckks_primes_below_bits": (I32, [U32, U32, U32, u64p]),
    "ckks_find_negacyclic_root": (U64, [U64, U32]),
    "ckks_is_prime": (I32, [U64]),
    "ckks_ctx_create": (I32, [U32, u64p, U32, u64p, U32, ctypes.POINTER(VP)]),
    "ckks_ctx_destroy": (I32, [VP]),
    "ckks_ctx_set_tensor_cores": (I32, [VP, I32]),
    "ckks_ctx_tensor_cores": (I32, [VP]),
    "ckks_ctx_last_mac_path": (I32, [VP]),
    "ckks_ctx_autotune": (I32, [VP, U32, U32, VP]),
    "ckks_ctx_tuning_report": (I32, [VP, ctypes.c_char_p, ctypes.c_uint64]),
    "ckks_ctx_psi": (I32, [VP, u64p]),
    "ckks_ntt_forward": (I32, [VP, VP, VP, U32, U32, U32, VP]),
    "ckks_ntt_inverse": (I32, [VP, VP, VP, U32, U32, U32, VP]),
    "ckks_ntt_forward_inplace_static": (I32, [VP, VP, U32, U32, U32, VP]),
    "ckks_ntt_forward_host": (I32, [VP, u64p, u64p, U32, U32, U32]),
    "ckks_ntt_inverse_host": (I32, [VP, u64p, u64p, U32, U32, U32]),
    "ckks_automorphism_coef": (I32, [VP, VP, VP, U32, U32, U32, U64, VP]),
    "ckks_automorphism_ntt": (I32, [VP, VP, VP, U32, U32, U32, U64, VP]),
    "ckks_rotation_exponent_left": (U64, [U32, U64]),
    "ckks_rotation_exponent_right": (U64, [U32, U64]),
    "ckks_conjugation_exponent": (U64, [U32]),
    "ckks_pointwise": (I32, [VP, VP, VP, VP, U32, U32, U32, I32, VP]),
    "ckks_rescale": (I32, [VP, VP, VP, U32, U32, VP]),
    "ckks_mod_down": (I32, [VP, VP, VP, U32, U32, VP]),
    "ckks_mod_switch": (I32, [VP, VP, VP, U32, U32, U32, VP]),
    "ckks_bounded_digit_count": (I32, [VP, U32, U32, ctypes.POINTER(U32)]),
    "ckks_bounded_decompose": (I32, [VP, VP, U32, U32, U32, VP, VP]),
    "ckks_bounded_digits_automorphism": (I32, [VP, VP, VP, U32, U32, U32, U64, VP]),
    "ckks_hybrid_key_generate": (I32, [VP, U32, U32, U64, i8p, U64, ctypes.c_double, ctypes.POINTER(VP)]),
    "ckks_hybrid_key_upload": (I32, [VP, U32, U32, U64, u64p, ctypes.POINTER(VP)]),
    "ckks_rnsblock_key_generate": (I32, [VP, U32, u32p, U32, U64, i8p, U64, ctypes.c_double, ctypes.POINTER(VP)]),
    "ckks_rnsblock_key_upload": (I32, [VP, U32, u32p, U32, U64, u64p, ctypes.POINTER(VP)]),
    "ckks_rns_key_generate": (I32, [VP, U32, u32p, U32, U64, i8p, U64, ctypes.c_double, ctypes.POINTER(VP)]),
    "ckks_rns_key_upload": (I32, [VP, U32, u32p, U32, U64, u64p, ctypes.POINTER(VP)]),
    "ckks_rns_relin_key_generate": (I32, [VP, U32, u32p, U32, i8p, U64, ctypes.c_double, ctypes.POINTER(VP)]),
    "ckks_rns_relin_key_upload": (I32, [VP, U32, u32p, U32, u64p, ctypes.POINTER(VP)]),
    "ckks_relin_key_generate": (I32, [VP, U32, U32, i8p, U64, ctypes.c_double, ctypes.POINTER(VP)]),
    "ckks_relin_key_upload": (I32, [VP, U32, U32, u64p, ctypes.POINTER(VP)]),
    "ckks_ksk_info": (I32, [VP, ctypes.POINTER(U32), ctypes.POINTER(U64)]),
    "ckks_ksk_download": (I32, [VP, u64p]),
    "ckks_ksk_destroy": (I32, [VP]),
    "ckks_rotate": (I32, [VP, VP, VP, VP, U32, VP]),
    "ckks_rotate_hoisted": (I32, [VP, ctypes.POINTER(VP), U32, VP, VP, U32, VP]),
    "ckks_rotate_hoisted_timed": (I32, [VP, ctypes.POINTER(VP), U32, VP, VP, U32, VP, ctypes.POINTER(ctypes.c_double)]),
    "ckks_rotate_hoisted_host": (I32, [VP, ctypes.POINTER(VP), U32, u64p, u64p, U32]),
    "ckks_tensor": (I32, [VP, VP, VP, VP, U32, U32, VP]),
    "ckks_relinearize": (I32, [VP, VP, VP, VP, U32, VP]),
    "ckks_multiply_relin_rescale": (I32, [VP, VP, VP, VP, VP, U32, VP]),
    "ckks_multiply_relin_rescale_host": (I32, [VP, VP, u64p, u64p, u64p, U32]),
    "ckks_mul_plain": (I32, [VP, VP, VP, VP, U32, U32, U32, VP]),
    "ckks_fft_stage": (I32, [VP, ctypes.POINTER(VP), U32, I32, VP, VP, VP, U32, U32, VP]),
    "ckks_diag_stage": (I32, [VP, ctypes.POINTER(VP), U32, I32, VP, VP, VP, U32, U32, I32, VP]),
    "ckks_ccmm_structured": (I32, [VP, VP, VP, VP, VP, U32, U32, U32, VP]),
    "ckks_fft_stage_multi": (I32, [VP, ctypes.POINTER(VP), U32, u32p, U32, VP, VP, U32, VP, U32, U32, VP]),
    "ckks_park_mod_pp_mm": (I32, [VP, VP, VP, U32, U32, U32, U64, VP]),
    "ckks_park_mod_pp_mm_host": (I32, [u64p, u64p, u64p, U32, U32, U32, U64]),
    "ckks_park_mod_pp_mm_with_backend": (I32, [VP, VP, VP, U32, U32, U32, U64, I32, VP]),
    "ckks_park_last_timing": (I32, [ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]),
    "ckks_rng_create": (I32, [U64, ctypes.POINTER(VP)]),
    "ckks_rng_create_from_seed": (I32, [ctypes.c_char_p, ctypes.POINTER(VP)]),
    "ckks_rng_destroy": (I32, [VP]),
    "ckks_rng_next_u32": (I32, [VP, u32p]),
    "ckks_rng_next_u64": (I32, [VP, u64p]),
    "ckks_rng_fill_u32": (I32, [VP, u32p, U64]),
    "ckks_rng_word_position": (I32, [VP, u64p]),
    "ckks_rng_ternary_secret": (I32, [VP, U32, i8p]),
    "ckks_rng_error": (I32, [VP, U32, I32, ctypes.c_double, ctypes.POINTER(ctypes.c_int64)]),
    "ckks_rng_uniform_residues": (I32, [VP, U32, U64, u64p]),
    "ckks_hybrid_key_generate_rng": (I32, [VP, U32, U32, U64, i8p, I32, ctypes.c_double, VP, ctypes.POINTER(VP)]),
    "ckks_relin_key_generate_rng": (I32, [VP, U32, U32, i8p, I32, ctypes.c_double, VP, ctypes.POINTER(VP)]),
    "ckks_encrypt_rng_host": (I32, [VP, U32, u64p, i8p, I32, ctypes.c_double, VP, u64p]),
    "ckks_encode": (I32, [VP, VP, VP, U32, U32, ctypes.c_double, VP]),
    "ckks_decode": (I32, [VP, VP, VP, U32, U32, ctypes.c_double, VP]),
}

STATUS = {0: "OK", -1: "BAD_ARG", -2: "BASIS_MISMATCH", -3: "EXPONENT_MISMATCH", -4: "OOM", -5: "CUDA",
          -6: "TIMEOUT", -7: "GADGET_CAPACITY"}

_lib = None


class CkksError(RuntimeError):
    def __init__(self, status, message):
        super().__init__("%s (%d): %s" % (STATUS.get(status, "?"), status, message))
        self.status = status


def build():
    import importlib.util
    spec = importlib.util.spec_from_file_location("ckks_b200_build", os.path.join(PKG, "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.build()


def lib():
    """Loads the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libckks_b200.so is not built; run __graft_entry__.build()")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc):
    if rc != 0:
        raise CkksError(rc, lib().ckks_last_error_string().decode())


def _u64(a):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.uint64))
    return a, a.ctypes.data_as(u64p)


def _dptr(t):
    """Device pointer of a contiguous CUDA tensor."""
    import torch
    assert t.is_cuda and t.is_contiguous(), "expected a contiguous CUDA tensor"
    return ctypes.c_void_p(t.data_ptr())


def _stream(stream):
    if stream is None:
        import torch
        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    return ctypes.c_void_p(stream)


def as_u64_tensor(a, device="cuda"):
    """numpy uint64 -> torch CUDA tensor holding the same bits (int64 view)."""
    import torch
    a = np.ascontiguousarray(np.asarray(a, dtype=np.uint64))
    return torch.from_numpy(a.view(np.int64)).to(device)


def to_numpy_u64(t):
    return t.detach().cpu().numpy().view(np.uint64)


class Context:
    """Device context: ring degree, Q limbs then P limbs, NTT tables."""

    def __init__(self, log_n, q, p=()):
        self.log_n = int(log_n)
        self.n = 1 << self.log_n
        self.q = [int(x) for x in q]
        self.p = [int(x) for x in p]
        qa, qp = _u64(self.q)
        pa, pp = _u64(self.p if self.p else [0])
        h = ctypes.c_void_p()
        check(lib().ckks_ctx_create(self.log_n, qp, len(self.q), pp, len(self.p), ctypes.byref(h)))
        self.handle = h

    @property
    def moduli(self):
        return self.q + self.p

    @property
    def psi(self):
        out = np.zeros(len(self.moduli), np.uint64)
        check(lib().ckks_ctx_psi(self.handle, out.ctypes.data_as(u64p)))
        return [int(x) for x in out]

    @property
    def tensor_cores(self):
        """True when bounded hoisted rotations run their key-switch MAC, and the
        structured CCMM its per-slot products (m, k <= 64), on the INT8 tensor
        cores (enabled by default where the device has them)."""
        return bool(lib().ckks_ctx_tensor_cores(self.handle))

    @tensor_cores.setter
    def tensor_cores(self, enable):
        check(lib().ckks_ctx_set_tensor_cores(self.handle, 1 if enable else 0))

    @property
    def last_mac_path(self):
        """Path of the most recent hoisted rotation MAC or CCMM slot product on
        this context: "tensor_cores", "cuda_cores" or None (neither ran yet)."""
        return {1: "tensor_cores", 0: "cuda_cores"}.get(int(lib().ckks_ctx_last_mac_path(self.handle)))

    def autotune(self, limbs, polys, stream=None):
        """Times the NTT passes' tile choices on a limbs x polys batch, keeps the
        fastest, and returns the record."""
        check(lib().ckks_ctx_autotune(self.handle, int(limbs), int(polys), _stream(stream)))
        return self.tuning_report

    @property
    def tuning_report(self):
        buf = ctypes.create_string_buffer(8192)
        check(lib().ckks_ctx_tuning_report(self.handle, buf, len(buf)))
        return buf.value.decode()

    def close(self):
        if getattr(self, "handle", None):
            lib().ckks_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ring/prepared_rns_ntt.rs:39-83 -- [n_polys][limbs][N] tensors
    def ntt_forward(self, data, limb_begin=0, out=None, stream=None):
        limbs = data.shape[-2]
        out = data if out is None else out
        check(lib().ckks_ntt_forward(self.handle, _dptr(data), _dptr(out), data.numel() // (limbs * self.n),
                                     limb_begin, limbs, _stream(stream)))
        return out

    def ntt_inverse(self, data, limb_begin=0, out=None, stream=None):
        limbs = data.shape[-2]
        out = data if out is None else out
        check(lib().ckks_ntt_inverse(self.handle, _dptr(data), _dptr(out), data.numel() // (limbs * self.n),
                                     limb_begin, limbs, _stream(stream)))
        return out

    def ntt_forward_host(self, data, limb_begin=0):
        a, ap = _u64(data)
        out = np.empty_like(a)
        limbs = a.shape[-2]
        check(lib().ckks_ntt_forward_host(self.handle, ap, out.ctypes.data_as(u64p), a.size // (limbs * self.n),
                                          limb_begin, limbs))
        return out

    def ntt_inverse_host(self, data, limb_begin=0):
        a, ap = _u64(data)
        out = np.empty_like(a)
        limbs = a.shape[-2]
        check(lib().ckks_ntt_inverse_host(self.handle, ap, out.ctypes.data_as(u64p), a.size // (limbs * self.n),
                                          limb_begin, limbs))
        return out


    # ---------------------------------------------------------- ring ops
    def automorphism_coef(self, data, exponent, limb_begin=0, out=None, stream=None):
        """ckks/automorphism.rs:8-48 over [n_polys][limbs][N]."""
        import torch
        limbs = data.shape[-2]
        out = torch.empty_like(data) if out is None else out
        check(lib().ckks_automorphism_coef(self.handle, _dptr(data), _dptr(out), data.numel() // (limbs * self.n),
                                           limb_begin, limbs, int(exponent), _stream(stream)))
        return out

    def automorphism_ntt(self, data, exponent, limb_begin=0, out=None, stream=None):
        """ring/ntt_galois_permutation.rs:5-19 over NTT-domain [n_polys][limbs][N]."""
        import torch
        limbs = data.shape[-2]
        out = torch.empty_like(data) if out is None else out
        check(lib().ckks_automorphism_ntt(self.handle, _dptr(data), _dptr(out), data.numel() // (limbs * self.n),
                                          limb_begin, limbs, int(exponent), _stream(stream)))
        return out

    def pointwise(self, a, b, op, limb_begin=0, out=None, stream=None):
        import torch
        limbs = a.shape[-2]
        out = torch.empty_like(a) if out is None else out
        check(lib().ckks_pointwise(self.handle, _dptr(a), _dptr(b), _dptr(out), a.numel() // (limbs * self.n),
                                   limb_begin, limbs, {"mul": 0, "add": 1, "sub": 2}[op], _stream(stream)))
        return out

    def rescale(self, data, stream=None):
        """ckks/rns_rescale.rs:107-167: [..., limbs, N] -> [..., limbs-1, N]."""
        import torch
        limbs = data.shape[-2]
        out = torch.empty(data.shape[:-2] + (limbs - 1, self.n), dtype=torch.int64, device=data.device)
        check(lib().ckks_rescale(self.handle, _dptr(data), _dptr(out), data.numel() // (limbs * self.n), limbs,
                                 _stream(stream)))
        return out

    def mod_switch(self, ct, limbs_out=None, stream=None):
        """ckks/rns_mod_switch.rs:14-58: [..., 2, limbs, N] -> [..., 2, limbs_out, N]
        keeping the leading limbs (default: one level down), scale unchanged."""
        import torch
        limbs = ct.shape[-2]
        limbs_out = limbs - 1 if limbs_out is None else int(limbs_out)
        out = torch.empty(ct.shape[:-2] + (limbs_out, self.n), dtype=torch.int64, device=ct.device)
        check(lib().ckks_mod_switch(self.handle, _dptr(ct), _dptr(out), ct.numel() // (2 * limbs * self.n), limbs,
                                    limbs_out, _stream(stream)))
        return out

    def mod_down(self, data, stream=None):
        """ring/auxiliary_modulus.rs:89-171: [..., q_limbs+K, N] -> [..., q_limbs, N]."""
        import torch
        q_limbs = data.shape[-2] - len(self.p)
        out = torch.empty(data.shape[:-2] + (q_limbs, self.n), dtype=torch.int64, device=data.device)
        check(lib().ckks_mod_down(self.handle, _dptr(data), _dptr(out), data.numel() // ((q_limbs + len(self.p)) * self.n),
                                  q_limbs, _stream(stream)))
        return out

    def digit_count(self, q_limbs, base_log):
        d = U32()
        check(lib().ckks_bounded_digit_count(self.handle, q_limbs, base_log, ctypes.byref(d)))
        return d.value

    def bounded_decompose(self, poly, base_log, stream=None):
        """grafting/bounded_gadget.rs:59-118: [..., q_limbs, N] -> int64 digits [..., D, N]."""
        import torch
        q_limbs = poly.shape[-2]
        npoly = poly.numel() // (q_limbs * self.n)
        D = self.digit_count(q_limbs, base_log)
        out = torch.empty(poly.shape[:-2] + (D, self.n), dtype=torch.int64, device=poly.device)
        check(lib().ckks_bounded_decompose(self.handle, _dptr(poly), npoly, q_limbs, base_log, _dptr(out),
                                           _stream(stream)))
        return out

    def bounded_digits_automorphism(self, digits, base_log, exponent, stream=None):
        import torch
        D = digits.shape[-2]
        out = torch.empty_like(digits)
        check(lib().ckks_bounded_digits_automorphism(self.handle, _dptr(digits), _dptr(out),
                                                     digits.numel() // (D * self.n), D, base_log, int(exponent),
                                                     _stream(stream)))
        return out

    def rotation_exponent_left(self, steps):
        return int(lib().ckks_rotation_exponent_left(self.n, int(steps)))

    def rotation_exponent_right(self, steps):
        return int(lib().ckks_rotation_exponent_right(self.n, int(steps)))


class ChaCha20Rng:
    """rand_chacha::ChaCha20Rng as the reference seeds and consumes it (host side).

    seed_from_u64 / from_seed, next_u32 / next_u64, and the reference's
    samplers: ternary secret (rlwe/secret_key.rs:25-40), errors
    (rlwe/error.rs:33-156: ErrorDistribution BoundedUniform or
    DiscreteGaussian) and uniform residues (rlwe/uniform.rs:12-30). Passing
    one instance through several calls continues one stream, as `&mut rng`
    does in the reference.
    """

    BOUNDED_UNIFORM, GAUSSIAN = 0, 1

    def __init__(self, handle):
        self.handle = handle

    @classmethod
    def seed_from_u64(cls, seed):
        h = ctypes.c_void_p()
        check(lib().ckks_rng_create(int(seed) & (2**64 - 1), ctypes.byref(h)))
        return cls(h)

    @classmethod
    def from_seed(cls, seed32):
        b = bytes(seed32)
        if len(b) != 32:
            raise ValueError("ChaCha20Rng seed must be 32 bytes")
        h = ctypes.c_void_p()
        check(lib().ckks_rng_create_from_seed(b, ctypes.byref(h)))
        return cls(h)

    def next_u32(self):
        v = U32()
        check(lib().ckks_rng_next_u32(self.handle, ctypes.byref(v)))
        return v.value

    def next_u64(self):
        v = U64()
        check(lib().ckks_rng_next_u64(self.handle, ctypes.byref(v)))
        return v.value

    def words(self, n):
        out = np.zeros(n, np.uint32)
        check(lib().ckks_rng_fill_u32(self.handle, out.ctypes.data_as(u32p), n))
        return out

    def word_position(self):
        v = U64()
        check(lib().ckks_rng_word_position(self.handle, ctypes.byref(v)))
        return v.value

    def ternary_secret(self, n):
        out = np.zeros(n, np.int8)
        check(lib().ckks_rng_ternary_secret(self.handle, n, out.ctypes.data_as(i8p)))
        return out

    def error(self, n, kind, param):
        out = np.zeros(n, np.int64)
        check(lib().ckks_rng_error(self.handle, n, kind, float(param),
                                   out.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))))
        return out

    def uniform_residues(self, n, modulus):
        out = np.zeros(n, np.uint64)
        check(lib().ckks_rng_uniform_residues(self.handle, n, int(modulus), out.ctypes.data_as(u64p)))
        return out

    def close(self):
        if getattr(self, "handle", None):
            lib().ckks_rng_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def encrypt_rng(ctx, q_limbs, message, secret, rng, kind=ChaCha20Rng.GAUSSIAN, param=3.2):
    """encrypt_rns_raw_with_distribution_ntt_rng (grafting/rns_key_switch.rs:245-387) on the
    reference's stream: message [q_limbs][N] coefficients -> ciphertext [2][q_limbs][N]."""
    m = np.ascontiguousarray(np.asarray(message, np.uint64))
    s = np.ascontiguousarray(np.asarray(secret, np.int8))
    out = np.zeros((2, q_limbs, ctx.n), np.uint64)
    check(lib().ckks_encrypt_rng_host(ctx.handle, q_limbs, m.ctypes.data_as(u64p), s.ctypes.data_as(i8p), kind,
                                      float(param), rng.handle, out.ctypes.data_as(u64p)))
    return out


PARK_BACKENDS = {"auto": 0, "tensor_cores": 1, "cuda_cores": 2}


def park_mod_pp_mm(lhs, rhs, modulus, out=None, stream=None, backend="auto"):
    """park_mod_pp_mm (ccmm/park.rs:1634-1647): (lhs x rhs) mod modulus.

    lhs, rhs: row-major u64 matrices as torch CUDA int64 tensors (device path)
    or numpy uint64 arrays (host path, synchronous, backend "auto").
    backend (device path): "auto" / "tensor_cores" (INT8 tcgen05 products of
    byte planes) / "cuda_cores" (192-bit exact sums); all give the same words,
    like the reference's ParkModPpMmBackend variants."""
    if backend not in PARK_BACKENDS:
        raise ValueError("park_mod_pp_mm: backend is one of %s" % sorted(PARK_BACKENDS))
    if isinstance(lhs, np.ndarray):
        a = np.ascontiguousarray(lhs, np.uint64); b = np.ascontiguousarray(rhs, np.uint64)
        if a.ndim != 2 or b.ndim != 2 or a.shape[1] != b.shape[0]:
            raise ValueError("park_mod_pp_mm: shapes do not chain")
        c = np.zeros((a.shape[0], b.shape[1]), np.uint64)
        check(lib().ckks_park_mod_pp_mm_host(a.ctypes.data_as(u64p), b.ctypes.data_as(u64p), c.ctypes.data_as(u64p),
                                             a.shape[0], a.shape[1], b.shape[1], int(modulus)))
        return c
    import torch
    if lhs.dim() != 2 or rhs.dim() != 2 or lhs.shape[1] != rhs.shape[0]:
        raise ValueError("park_mod_pp_mm: shapes do not chain")
    if not (lhs.is_contiguous() and rhs.is_contiguous()):
        raise ValueError("park_mod_pp_mm: operands must be contiguous")
    out = torch.empty((lhs.shape[0], rhs.shape[1]), dtype=torch.int64, device=lhs.device) if out is None else out
    check(lib().ckks_park_mod_pp_mm_with_backend(_dptr(lhs), _dptr(rhs), _dptr(out), lhs.shape[0], lhs.shape[1],
                                                 rhs.shape[1], int(modulus), PARK_BACKENDS[backend],
                                                 _stream(stream)))
    return out


def park_last_timing():
    """(pack ms, GEMM ms) of this thread's last tensor-core Park call (CUDA events)."""
    p, g = ctypes.c_float(), ctypes.c_float()
    check(lib().ckks_park_last_timing(ctypes.byref(p), ctypes.byref(g)))
    return p.value, g.value


class KeySwitchKey:
    """A key-switching key resident in HBM (ckks_ksk)."""

    HYBRID_BOUNDED, HYBRID_RNS_BLOCK, RELIN_BOUNDED, RNS_BLOCK, RELIN_RNS_BLOCK = 0, 1, 2, 3, 4

    def __init__(self, ctx, handle, kind, q_limbs, exponent=1, base_log=0, blocks=()):
        self.ctx, self.handle, self.kind = ctx, handle, kind
        self.q_limbs, self.exponent, self.base_log, self.blocks = q_limbs, exponent, base_log, tuple(blocks)

    @staticmethod
    def _secret(secret):
        s = np.ascontiguousarray(np.asarray(secret, dtype=np.int8))
        return s, s.ctypes.data_as(i8p)

    @classmethod
    def hybrid_generate(cls, ctx, q_limbs, base_log, exponent, secret, seed, sigma=3.2):
        """PreparedHybridRnsGaloisKey::generate_with_distribution_ntt_rng (hybrid_rns_galois_key.rs:61-170)."""
        s, sp = cls._secret(secret)
        h = ctypes.c_void_p()
        check(lib().ckks_hybrid_key_generate(ctx.handle, q_limbs, base_log, int(exponent), sp, seed, sigma,
                                             ctypes.byref(h)))
        return cls(ctx, h, cls.HYBRID_BOUNDED, q_limbs, exponent, base_log)

    @classmethod
    def hybrid_generate_rng(cls, ctx, q_limbs, base_log, exponent, secret, rng, kind=ChaCha20Rng.GAUSSIAN,
                            param=3.2):
        """generate_with_distribution_ntt_rng on the reference's ChaCha20 stream (rng continues)."""
        s, sp = cls._secret(secret)
        h = ctypes.c_void_p()
        check(lib().ckks_hybrid_key_generate_rng(ctx.handle, q_limbs, base_log, int(exponent), sp, kind, float(param),
                                                 rng.handle, ctypes.byref(h)))
        return cls(ctx, h, cls.HYBRID_BOUNDED, q_limbs, exponent, base_log)

    @classmethod
    def hybrid_upload(cls, ctx, q_limbs, base_log, exponent, entries):
        e, ep = _u64(entries)
        h = ctypes.c_void_p()
        check(lib().ckks_hybrid_key_upload(ctx.handle, q_limbs, base_log, int(exponent), ep, ctypes.byref(h)))
        return cls(ctx, h, cls.HYBRID_BOUNDED, q_limbs, exponent, base_log)

    @classmethod
    def rnsblock_generate(cls, ctx, q_limbs, blocks, exponent, secret, seed, sigma=3.2):
        s, sp = cls._secret(secret)
        b = np.ascontiguousarray(np.asarray(blocks, np.uint32))
        h = ctypes.c_void_p()
        check(lib().ckks_rnsblock_key_generate(ctx.handle, q_limbs, b.ctypes.data_as(u32p), len(b), int(exponent), sp,
                                               seed, sigma, ctypes.byref(h)))
        return cls(ctx, h, cls.HYBRID_RNS_BLOCK, q_limbs, exponent, 0, blocks)

    @classmethod
    def rnsblock_upload(cls, ctx, q_limbs, blocks, exponent, entries):
        e, ep = _u64(entries)
        b = np.ascontiguousarray(np.asarray(blocks, np.uint32))
        h = ctypes.c_void_p()
        check(lib().ckks_rnsblock_key_upload(ctx.handle, q_limbs, b.ctypes.data_as(u32p), len(b), int(exponent), ep,
                                             ctypes.byref(h)))
        return cls(ctx, h, cls.HYBRID_RNS_BLOCK, q_limbs, exponent, 0, blocks)

    @classmethod
    def rns_generate(cls, ctx, q_limbs, blocks, exponent, secret, seed, sigma=3.2):
        """Ordinary RNS Galois key without auxiliary limbs: PreparedRnsGaloisKey
        (ckks/rns_galois_key.rs, grafting/rns_key_switch.rs:1155-1258)."""
        s, sp = cls._secret(secret)
        b = np.ascontiguousarray(np.asarray(blocks, np.uint32))
        h = ctypes.c_void_p()
        check(lib().ckks_rns_key_generate(ctx.handle, q_limbs, b.ctypes.data_as(u32p), len(b), int(exponent), sp,
                                          seed, sigma, ctypes.byref(h)))
        return cls(ctx, h, cls.RNS_BLOCK, q_limbs, exponent, 0, blocks)

    @classmethod
    def rns_upload(cls, ctx, q_limbs, blocks, exponent, entries):
        """NTT-domain entries [dnum][q_limbs][2][N] (the reference's PreparedRnsKeySwitchKey)."""
        e, ep = _u64(entries)
        b = np.ascontiguousarray(np.asarray(blocks, np.uint32))
        h = ctypes.c_void_p()
        check(lib().ckks_rns_key_upload(ctx.handle, q_limbs, b.ctypes.data_as(u32p), len(b), int(exponent), ep,
                                        ctypes.byref(h)))
        return cls(ctx, h, cls.RNS_BLOCK, q_limbs, exponent, 0, blocks)

    @classmethod
    def rns_relin_generate(cls, ctx, q_limbs, blocks, secret, seed, sigma=3.2):
        """RNS-block relinearization key (RnsMultiplicationKey, target s^2)."""
        s, sp = cls._secret(secret)
        b = np.ascontiguousarray(np.asarray(blocks, np.uint32))
        h = ctypes.c_void_p()
        check(lib().ckks_rns_relin_key_generate(ctx.handle, q_limbs, b.ctypes.data_as(u32p), len(b), sp, seed, sigma,
                                                ctypes.byref(h)))
        return cls(ctx, h, cls.RELIN_RNS_BLOCK, q_limbs, 1, 0, blocks)

    @classmethod
    def rns_relin_upload(cls, ctx, q_limbs, blocks, entries):
        """Coefficient-domain entries [dnum][2][q_limbs][N]."""
        e, ep = _u64(entries)
        b = np.ascontiguousarray(np.asarray(blocks, np.uint32))
        h = ctypes.c_void_p()
        check(lib().ckks_rns_relin_key_upload(ctx.handle, q_limbs, b.ctypes.data_as(u32p), len(b), ep,
                                              ctypes.byref(h)))
        return cls(ctx, h, cls.RELIN_RNS_BLOCK, q_limbs, 1, 0, blocks)

    @classmethod
    def relin_generate(cls, ctx, q_limbs, base_log, secret, seed, sigma=3.2):
        """BoundedRnsMultiplicationKey::generate_with_distribution_ntt_rng (bounded_key_switch.rs:28-104)."""
        s, sp = cls._secret(secret)
        h = ctypes.c_void_p()
        check(lib().ckks_relin_key_generate(ctx.handle, q_limbs, base_log, sp, seed, sigma, ctypes.byref(h)))
        return cls(ctx, h, cls.RELIN_BOUNDED, q_limbs, 1, base_log)

    @classmethod
    def relin_generate_rng(cls, ctx, q_limbs, base_log, secret, rng, kind=ChaCha20Rng.GAUSSIAN, param=3.2):
        """BoundedRnsMultiplicationKey::generate_with_distribution_ntt_rng on the reference's stream."""
        s, sp = cls._secret(secret)
        h = ctypes.c_void_p()
        check(lib().ckks_relin_key_generate_rng(ctx.handle, q_limbs, base_log, sp, kind, float(param), rng.handle,
                                                ctypes.byref(h)))
        return cls(ctx, h, cls.RELIN_BOUNDED, q_limbs, 1, base_log)

    @classmethod
    def relin_upload(cls, ctx, q_limbs, base_log, entries):
        e, ep = _u64(entries)
        h = ctypes.c_void_p()
        check(lib().ckks_relin_key_upload(ctx.handle, q_limbs, base_log, ep, ctypes.byref(h)))
        return cls(ctx, h, cls.RELIN_BOUNDED, q_limbs, 1, base_log)

    def info(self):
        d, w = U32(), U64()
        check(lib().ckks_ksk_info(self.handle, ctypes.byref(d), ctypes.byref(w)))
        return d.value, w.value

    def download(self):
        D, words = self.info()
        out = np.zeros(words, np.uint64)
        check(lib().ckks_ksk_download(self.handle, out.ctypes.data_as(u64p)))
        return out

    def close(self):
        if getattr(self, "handle", None):
            lib().ckks_ksk_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def rotate(ctx, key, ct, out=None, stream=None):
    """Key-switched Galois automorphism of [n_ct][2][q_limbs][N] ciphertexts
    (apply_hybrid_rns_galois_automorphism_with_prepared_ntt, hybrid_rns_galois_key.rs:293)."""
    import torch
    out = torch.empty_like(ct) if out is None else out
    n_ct = ct.numel() // (2 * key.q_limbs * ctx.n)
    check(lib().ckks_rotate(ctx.handle, key.handle, _dptr(ct), _dptr(out), n_ct, _stream(stream)))
    return out


def rotate_hoisted(ctx, keys, ct, out=None, stream=None):
    """Hoisted rotations: out [n_ct][n_keys][2][q_limbs][N]."""
    import torch
    q_limbs = keys[0].q_limbs
    n_ct = ct.numel() // (2 * q_limbs * ctx.n)
    if out is None:
        out = torch.empty((n_ct, len(keys), 2, q_limbs, ctx.n), dtype=torch.int64, device=ct.device)
    arr = (VP * len(keys))(*[k.handle.value for k in keys])
    check(lib().ckks_rotate_hoisted(ctx.handle, arr, len(keys), _dptr(ct), _dptr(out), n_ct, _stream(stream)))
    return out


ROTATION_PHASES = {0: "decompose+digit/base NTT", 2: "correction lists", 3: "key-switch MAC", 4: "inverse NTT",
                   5: "ModDown+sigma"}


def rotate_hoisted_timed(ctx, keys, ct, out=None, stream=None):
    """rotate_hoisted plus per-phase device milliseconds {phase name: ms}."""
    import torch
    q_limbs = keys[0].q_limbs
    n_ct = ct.numel() // (2 * q_limbs * ctx.n)
    if out is None:
        out = torch.empty((n_ct, len(keys), 2, q_limbs, ctx.n), dtype=torch.int64, device=ct.device)
    arr = (VP * len(keys))(*[k.handle.value for k in keys])
    ms = (ctypes.c_double * 8)()
    check(lib().ckks_rotate_hoisted_timed(ctx.handle, arr, len(keys), _dptr(ct), _dptr(out), n_ct, _stream(stream), ms))
    return out, {name: ms[i] for i, name in ROTATION_PHASES.items()}


def rotate_hoisted_host(ctx, keys, ct_host, out_host=None):
    a, ap = _u64(ct_host)
    q_limbs = keys[0].q_limbs
    n_ct = a.size // (2 * q_limbs * ctx.n)
    if out_host is None:
        out_host = np.empty((n_ct, len(keys), 2, q_limbs, ctx.n), np.uint64)
    arr = (VP * len(keys))(*[k.handle.value for k in keys])
    check(lib().ckks_rotate_hoisted_host(ctx.handle, arr, len(keys), ap, out_host.ctypes.data_as(u64p), n_ct))
    return out_host


class PreparedRnsNttPlan:
    """Mirror of ring/prepared_rns_ntt.rs: forward/inverse over a limb range."""

    def __init__(self, ctx, limb_begin=0, limb_count=None):
        self.ctx = ctx
        self.limb_begin = limb_begin
        self.limb_count = len(ctx.moduli) - limb_begin if limb_count is None else limb_count

    def forward(self, data, out=None):
        assert data.shape[-2] == self.limb_count
        return self.ctx.ntt_forward(data, self.limb_begin, out)

    def inverse(self, data, out=None):
        assert data.shape[-2] == self.limb_count
        return self.ctx.ntt_inverse(data, self.limb_begin, out)


# ------------------------------------------------------------ products
def _n_ct(ctx, t, polys, limbs):
    return t.numel() // (polys * limbs * ctx.n)


def tensor(ctx, lhs, rhs, out=None, stream=None):
    """rns_tensor_with_ntt (grafting/rns_key_switch.rs:1675-1722):
    [n][2][L][N] x [n][2][L][N] -> quadratic [n][3][L][N], coefficient domain."""
    import torch
    L = lhs.shape[-2]
    n_ct = _n_ct(ctx, lhs, 2, L)
    if out is None:
        out = torch.empty((n_ct, 3, L, ctx.n), dtype=torch.int64, device=lhs.device)
    check(lib().ckks_tensor(ctx.handle, _dptr(lhs), _dptr(rhs), _dptr(out), n_ct, L, _stream(stream)))
    return out


def relinearize(ctx, key, quad, out=None, stream=None):
    """bounded_rns_relinearize_with_ntt (grafting/bounded_key_switch.rs:139-223):
    [n][3][L][N] -> [n][2][L][N]."""
    import torch
    L = key.q_limbs
    n_ct = _n_ct(ctx, quad, 3, L)
    if out is None:
        out = torch.empty((n_ct, 2, L, ctx.n), dtype=torch.int64, device=quad.device)
    check(lib().ckks_relinearize(ctx.handle, key.handle, _dptr(quad), _dptr(out), n_ct, _stream(stream)))
    return out


def multiply_relinearize_rescale(ctx, key, lhs, rhs, out=None, stream=None):
    """multiply_relinearize_rescale_rns_ckks_bounded_with_ntt (ckks/rns_multiply.rs:262-300):
    [n][2][L][N] x [n][2][L][N] -> [n][2][L-1][N]."""
    import torch
    L = key.q_limbs
    n_ct = _n_ct(ctx, lhs, 2, L)
    if out is None:
        out = torch.empty((n_ct, 2, L - 1, ctx.n), dtype=torch.int64, device=lhs.device)
    check(lib().ckks_multiply_relin_rescale(ctx.handle, key.handle, _dptr(lhs), _dptr(rhs), _dptr(out), n_ct,
                                            _stream(stream)))
    return out


def multiply_relinearize_rescale_host(ctx, key, lhs, rhs):
    a, ap = _u64(lhs)
    b, bp = _u64(rhs)
    L = key.q_limbs
    n_ct = a.size // (2 * L * ctx.n)
    out = np.empty((n_ct, 2, L - 1, ctx.n), np.uint64)
    check(lib().ckks_multiply_relin_rescale_host(ctx.handle, key.handle, ap, bp, out.ctypes.data_as(u64p), n_ct))
    return out


def multiply_plain(ctx, ct, plain_ntt, out=None, stream=None):
    """multiply_plain_rns_ckks_with_prepared_ntt (ckks/rns_plain_multiply.rs:193-260):
    ct [n][2][L][N] times the NTT-domain plaintext [L][N] (shared) or [n][L][N]."""
    import torch
    L = ct.shape[-2]
    n_ct = _n_ct(ctx, ct, 2, L)
    n_plain = plain_ntt.numel() // (L * ctx.n)
    out = torch.empty_like(ct) if out is None else out
    check(lib().ckks_mul_plain(ctx.handle, _dptr(ct), _dptr(plain_ntt), _dptr(out), n_ct, L, n_plain, _stream(stream)))
    return out


def fft_stage(ctx, keys, diag_ntt, ct, identity=True, out=None, stream=None):
    """apply_stage (eblas/prepared_radix4_fft256.rs:744-822): rotations by
    `keys` (one per nonzero offset) times their NTT-prepared diagonals, plus
    the offset-0 diagonal times the input when `identity`, summed and
    rescaled. diag_ntt [len(keys) + identity][L][N]; ct [n][2][L][N] ->
    [n][2][L-1][N]."""
    import torch
    L = ct.shape[-2]
    n_ct = _n_ct(ctx, ct, 2, L)
    if out is None:
        out = torch.empty((n_ct, 2, L - 1, ctx.n), dtype=torch.int64, device=ct.device)
    arr = (VP * max(1, len(keys)))(*[k.handle.value for k in keys])
    check(lib().ckks_fft_stage(ctx.handle, arr, len(keys), 1 if identity else 0, _dptr(diag_ntt), _dptr(ct),
                               _dptr(out), n_ct, L, _stream(stream)))
    return out


def diag_stage(ctx, keys, diag_ntt, ct, identity=True, rescale=True, out=None, stream=None):
    """fft_stage with the rescale optional; with keys (rotate left by r, rotate
    right by r) and the identity term it is the packed radix-2 DIF FFT2 stage
    (eblas/fft.rs:3378-3470, fused-rescale form :3906-4000)."""
    import torch
    L = ct.shape[-2]
    n_ct = _n_ct(ctx, ct, 2, L)
    lo = L - 1 if rescale else L
    if out is None:
        out = torch.empty((n_ct, 2, lo, ctx.n), dtype=torch.int64, device=ct.device)
    arr = (VP * max(1, len(keys)))(*[k.handle.value for k in keys])
    check(lib().ckks_diag_stage(ctx.handle, arr, len(keys), 1 if identity else 0, _dptr(diag_ntt), _dptr(ct),
                                _dptr(out), n_ct, L, 1 if rescale else 0, _stream(stream)))
    return out


def matmul_structured(ctx, key, A, B, m, k, n, out=None, stream=None):
    """matmul_structured_bounded_with_ntt (matrix/rns_ckks_ciphertext.rs:204-318):
    A [k][m][2][L][N] and B [n][k][2][L][N] column-major ciphertext matrices ->
    C [n][m][2][L-1][N]."""
    import torch
    L = key.q_limbs
    if out is None:
        out = torch.empty((n, m, 2, L - 1, ctx.n), dtype=torch.int64, device=A.device)
    check(lib().ckks_ccmm_structured(ctx.handle, key.handle, _dptr(A), _dptr(B), _dptr(out), m, k, n,
                                     _stream(stream)))
    return out


def fft_stage_multi(ctx, keys, terms, diag_ntt, cts, n_out, out=None, stream=None):
    """Diagonal stage over several ciphertexts: out[a] = Rescale(sum over terms
    (a, src, key) of diag * rotate(cts[src], keys[key])); key == len(keys)
    selects the unrotated input. diag_ntt [len(terms)][L][N] in term order."""
    import torch
    L = cts.shape[-2]
    n_in = _n_ct(ctx, cts, 2, L)
    t = np.ascontiguousarray(np.asarray(terms, dtype=np.uint32).reshape(-1, 3))
    if out is None:
        out = torch.empty((n_out, 2, L - 1, ctx.n), dtype=torch.int64, device=cts.device)
    arr = (VP * max(1, len(keys)))(*[k.handle.value for k in keys])
    check(lib().ckks_fft_stage_multi(ctx.handle, arr, len(keys), t.ctypes.data_as(u32p), len(t), _dptr(diag_ntt),
                                     _dptr(cts), n_in, _dptr(out), n_out, L, _stream(stream)))
    return out


# ----------------------------------------------------- encode / decode
def encode(ctx, slots, q_limbs, scale, stream=None):
    """encode_rns (application_support/ckks.rs:39-62): complex slots [..., N/2]
    (numpy or a complex128 CUDA tensor) -> plaintexts [..., q_limbs, N] on the GPU."""
    import torch
    if isinstance(slots, np.ndarray):
        slots = torch.from_numpy(np.ascontiguousarray(slots, dtype=np.complex128)).cuda()
    slots = slots.contiguous()
    lead = tuple(slots.shape[:-1])
    n_msg = int(np.prod(lead)) if lead else 1
    out = torch.empty(lead + (q_limbs, ctx.n), dtype=torch.int64, device=slots.device)
    check(lib().ckks_encode(ctx.handle, _dptr(slots), _dptr(out), n_msg, q_limbs, float(scale), _stream(stream)))
    return out


def decode(ctx, poly, scale, stream=None):
    """Decode of application_support/ckks.rs:106-130: plaintexts [..., q_limbs, N]
    -> complex128 slots [..., N/2] (CUDA tensor)."""
    import torch
    q_limbs = poly.shape[-2]
    lead = tuple(poly.shape[:-2])
    n_msg = int(np.prod(lead)) if lead else 1
    out = torch.empty(lead + (ctx.n // 2,), dtype=torch.complex128, device=poly.device)
    check(lib().ckks_decode(ctx.handle, _dptr(poly), _dptr(out), n_msg, q_limbs, float(scale), _stream(stream)))
    return out
