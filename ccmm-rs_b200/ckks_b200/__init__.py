"""Python mirror of the ccmm-rs evaluation interface over libckks_b200.so.

The compute path is the sm_100a CUDA library behind the C ABI in
include/ckks_b200.h; this module only marshals torch CUDA tensors (device
memory) and host numpy arrays into those calls. There is no CPU fallback: if
the library or a GPU is missing, calls raise.

Names follow the reference crate (ring/, ckks/, grafting/):
  RnsNttPlan / PreparedRnsNttPlan    ring/rns_ntt.rs, ring/prepared_rns_ntt.rs
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

_SIGS = {
    "ckks_last_error_string": (ctypes.c_char_p, []),
    "ckks_version": (ctypes.c_char_p, []),
    "ckks_primes_below_bits": (I32, [U32, U32, U32, u64p]),
    "ckks_find_negacyclic_root": (U64, [U64, U32]),
    "ckks_is_prime": (I32, [U64]),
    "ckks_ctx_create": (I32, [U32, u64p, U32, u64p, U32, ctypes.POINTER(VP)]),
    "ckks_ctx_destroy": (I32, [VP]),
    "ckks_ctx_psi": (I32, [VP, u64p]),
    "ckks_ntt_forward": (I32, [VP, VP, VP, U32, U32, U32, VP]),
    "ckks_ntt_inverse": (I32, [VP, VP, VP, U32, U32, U32, VP]),
    "ckks_ntt_forward_host": (I32, [VP, u64p, u64p, U32, U32, U32]),
    "ckks_ntt_inverse_host": (I32, [VP, u64p, u64p, U32, U32, U32]),
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
