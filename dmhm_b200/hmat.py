"""Python mirror of the reference's serial H-matrix API over the C ABI.

Names, argument meaning and error behaviour follow YingzhouLi/dmhm's
``HMat2d<double>`` / ``HMat3d<double>`` (include/dmhm/hmat2d.hpp:22-393,
include/dmhm/hmat3d.hpp) and the globals of src/core/global.cpp, so code
written against the reference reads the same:

    Initialize(); SetOversample(4)
    H = HMat2d(S, numLevels, maxRank, stronglyAdmissible, xSize, ySize)
    y = H.Multiply(1.0, x)            # vector or dense (numpy or CUDA tensor)
    C = H.Multiply(1.0, B_hmat)       # H*H with randomized compression
    H.SchulzInvert(-1)

Every numeric operation runs in the sm_100a kernels of ``libdmhm_b200.so``;
nothing here computes.  Vectors are in hierarchical ordering.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import check, lib

LCG_SEED = (21 << 32) | 17


@dataclass
class Sparse:
    """CSR matrix (include/dmhm/core/sparse.hpp:16-28), hierarchical order."""
    height: int
    width: int
    rowOffsets: np.ndarray
    columnIndices: np.ndarray
    nonzeros: np.ndarray
    symmetric: bool = False


class Context:
    """Device, CUDA stream, generators and Oversample() of one engine instance."""

    def __init__(self, device: int = 0, stream: Optional[int] = None):
        h = C.c_void_p()
        check(lib().hm_context_create(int(device), C.c_void_p(stream or 0), C.byref(h)))
        self._h = h
        self.device = device

    @property
    def handle(self):
        return self._h

    def synchronize(self):
        check(lib().hm_context_synchronize(self._h))

    def set_oversample(self, p: int):
        check(lib().hm_set_oversample(self._h, int(p)))

    def oversample(self) -> int:
        v = C.c_int()
        check(lib().hm_get_oversample(self._h, C.byref(v)))
        return v.value

    def set_compression_tolerance(self, tol: float):
        check(lib().hm_set_compression_tolerance(self._h, float(tol)))

    def set_low_precision(self, on: bool):
        """Low-precision phase for this context's H*H products: range samples
        on the TF32 tensor cores, block roundings in FP32."""
        check(lib().hm_set_low_precision(self._h, int(bool(on))))

    def compression_tolerance(self) -> float:
        v = C.c_double()
        check(lib().hm_get_compression_tolerance(self._h, C.byref(v)))
        return v.value

    # -- learned sample counts ------------------------------------------------
    def use_rank_model(self, model, margin: int = 2, probes: int = 4):
        """Attach a RankModel to the H*H compressions (None detaches)."""
        check(lib().hm_use_rank_model(self._h, model.handle if model is not None else None,
                                      int(margin), int(probes)))

    def rank_log_enable(self, on: bool = True):
        check(lib().hm_rank_log_enable(self._h, 1 if on else 0))

    def rank_log(self, clear: bool = False):
        """(features [n x F] float32, kept-rank fractions [n] float32)."""
        import numpy as np
        n = C.c_int()
        check(lib().hm_rank_log_read(self._h, None, None, 0, C.byref(n), 0))
        F = lib().hm_rank_feature_count()
        x = np.zeros((n.value, F), dtype=np.float32)
        t = np.zeros(n.value, dtype=np.float32)
        check(lib().hm_rank_log_read(self._h, x.ctypes.data_as(C.POINTER(C.c_float)),
                                     t.ctypes.data_as(C.POINTER(C.c_float)), n.value,
                                     C.byref(n), 1 if clear else 0))
        return x, t

    def rank_stats(self) -> dict:
        v = [C.c_int64() for _ in range(4)]
        check(lib().hm_rank_stats(self._h, *[C.byref(x) for x in v]))
        return {"compressions": v[0].value, "samples": v[1].value,
                "samples_plain": v[2].value, "fallbacks": v[3].value}

    def lcg_states(self):
        s, p = C.c_uint64(), C.c_uint64()
        check(lib().hm_get_lcg_states(self._h, C.byref(s), C.byref(p)))
        return s.value, p.value

    def set_lcg_states(self, serial: int, parallel: int):
        check(lib().hm_set_lcg_states(self._h, C.c_uint64(serial), C.c_uint64(parallel)))

    def close(self):
        if getattr(self, "_h", None):
            lib().hm_context_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_ctx: Optional[Context] = None


def Initialize(device: int = 0) -> Context:
    """Initialize (src/core/global.cpp:43-94): a context whose serial and
    parallel generators start at the reference seed {17, 21}."""
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(device)
    return _default_ctx


def Finalize():
    global _default_ctx
    if _default_ctx is not None:
        _default_ctx.close()
        _default_ctx = None


def _ctx(ctx: Optional[Context]) -> Context:
    return ctx if ctx is not None else Initialize()


def SetOversample(p: int, ctx: Optional[Context] = None):
    """SetOversample (global.cpp:155-159)."""
    _ctx(ctx).set_oversample(p)


def Oversample(ctx: Optional[Context] = None) -> int:
    """Oversample (global.cpp:152-153)."""
    return _ctx(ctx).oversample()


_DIST_TOL = [1e-16]   # compressionTolDouble (src/core/global.cpp:34)


def SetCompressionTolerance(tol: float):
    """SetCompressionTolerance (global.cpp:160-181): the relative tolerance
    of the DistHMat2d / DistHMat3d products.  As in the reference it leaves
    HMat2d / HMat3d at their fixed rank; ``Context.set_compression_tolerance``
    applies a tolerance to every product of one context."""
    if not 0.0 <= tol < 1.0:
        raise _lib.HMError(1, "compression tolerance must be in [0, 1)")
    _DIST_TOL[0] = float(tol)


def CompressionTolerance() -> float:
    return _DIST_TOL[0]


class _ScopedTolerance:
    def __init__(self, ctx: "Context", tol: float):
        self.ctx, self.tol = ctx, tol

    def __enter__(self):
        self.old = self.ctx.compression_tolerance()
        self.ctx.set_compression_tolerance(self.tol)

    def __exit__(self, *exc):
        self.ctx.set_compression_tolerance(self.old)


def _as_i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def natural_to_hierarchical_map(sizes: Sequence[int], num_levels: int) -> np.ndarray:
    """BuildNaturalToHierarchicalMap (src/HMat2d/HMat2d.cpp:69-87,
    src/HMat3d/HMat3d.cpp:91-110), computed by the library."""
    sz = _as_i32(list(sizes))
    out = np.empty(int(np.prod(sizes)), dtype=np.int32)
    check(lib().hm_natural_to_hierarchical_map(
        len(sizes), sz.ctypes.data_as(_lib._PI), int(num_levels), out.ctypes.data_as(_lib._PI)))
    return out


def _is_cuda_tensor(x) -> bool:
    return hasattr(x, "is_cuda") and bool(getattr(x, "is_cuda"))


class _HMatBase:
    """Common part of HMat2d / HMat3d: a handle to one device-resident H-matrix."""
    dim = 2

    def __init__(self, S: Optional[Sparse] = None, numLevels: int = 1, maxRank: int = 0,
                 stronglyAdmissible: bool = True, *sizes, ctx: Optional[Context] = None,
                 _handle=None):
        self.ctx = _ctx(ctx)
        self._h = None
        if _handle is not None:
            self._h = _handle
            return
        if S is None:
            return       # empty H-matrix (HMat2d(), hmat2d.hpp:40), filled by CopyFrom etc.
        if len(sizes) != self.dim:
            raise ValueError(f"expected {self.dim} grid sizes")
        if S.symmetric:
            raise _lib.HMError(4, "symmetric sparse storage builds NODE_SYMMETRIC blocks, "
                                  "which the H*H product and inversion do not support")
        N = int(np.prod(sizes))
        if S.height != N or S.width != N:
            raise _lib.HMError(1, "sparse matrix does not match the grid")
        rows = np.ascontiguousarray(S.rowOffsets, dtype=np.int64)
        cols = np.ascontiguousarray(S.columnIndices, dtype=np.int32)
        sz = _as_i32(list(sizes))
        h = C.c_void_p()
        if np.iscomplexobj(S.nonzeros):
            # HMat2d<std::complex<double>>: interleaved (re, im) values
            vals = np.ascontiguousarray(S.nonzeros, dtype=np.complex128).view(np.float64)
            create = lib().hm_create_from_csr_complex
        else:
            vals = np.ascontiguousarray(S.nonzeros, dtype=np.float64)
            create = lib().hm_create_from_csr
        check(create(
            self.ctx.handle, self.dim, sz.ctypes.data_as(_lib._PI), int(numLevels),
            int(maxRank), int(bool(stronglyAdmissible)), rows.ctypes.data_as(_lib._PI64),
            cols.ctypes.data_as(_lib._PI32), vals.ctypes.data_as(_lib._PD), C.byref(h)))
        self._h = h

    # -- lifetime -------------------------------------------------------------
    def __del__(self):
        try:
            if self._h:
                lib().hm_destroy(self._h)
                self._h = None
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    # -- AbstractHMat fulfilment (include/dmhm/core/abstract_hmat.hpp:20-40) ---
    def _info(self):
        h, w, L, r = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        counts = (C.c_int64 * 4)()
        nbytes = C.c_int64()
        check(lib().hm_info(self._h, C.byref(h), C.byref(w), C.byref(L), C.byref(r),
                            counts, C.byref(nbytes)))
        return h.value, w.value, L.value, r.value, list(counts), nbytes.value

    @property
    def is_complex(self) -> bool:
        """Scalar = std::complex<double> (stored in real form on the device)."""
        v = C.c_int()
        check(lib().hm_is_complex(self._h, C.byref(v)))
        return bool(v.value)

    def Height(self) -> int:
        h = self._info()[0]
        return h // 2 if self.is_complex else h

    def Width(self) -> int:
        w = self._info()[1]
        return w // 2 if self.is_complex else w

    def NumLevels(self) -> int:
        return self._info()[2]

    def MaxRank(self) -> int:
        return self._info()[3]

    def Symmetric(self) -> bool:
        return False

    def BlockCensus(self) -> dict:
        _, _, _, _, c, nbytes = self._info()
        return {"node": c[0], "low_rank": c[1], "dense": c[2], "rank_sum": c[3],
                "bytes": nbytes}

    def SampleRank(self, approxRank: int) -> int:
        """SampleRank (hmat2d.hpp:32-33)."""
        return approxRank + self.ctx.oversample()

    # -- one low-rank approximation of a product (hmat_tools) ---------------
    def LowRankProduct(self, alpha: float, B: "_HMatBase", sampleRank: int = None,
                       op: int = 0):
        """F ~= alpha op(A) B as (U, V) with F = U V^T: hmat_tools::Multiply
        (op 0), TransposeMultiply (op 1), AdjointMultiply (op 2)
        (include/dmhm/hmat_tools.hpp:1657-2152).  sampleRank defaults to
        SampleRank(min(A.MaxRank(), B.MaxRank()))."""
        n = self.Height()
        r = min(self.MaxRank(), B.MaxRank(), n)
        if sampleRank is None:
            sampleRank = self.SampleRank(r)
        U = np.zeros((n, max(r, 1)), order="F")
        V = np.zeros((n, max(r, 1)), order="F")
        rk = C.c_int()
        check(lib().hm_low_rank_product(self._h, int(op), float(alpha), B.handle, int(sampleRank),
                                        U.ctypes.data_as(_lib._PD), n, V.ctypes.data_as(_lib._PD),
                                        n, max(r, 1), C.byref(rk)))
        return U[:, :rk.value].copy(), V[:, :rk.value].copy()

    # -- wire format (src/HMat2d/Pack-incl.hpp) -------------------------------
    def PackedSize(self) -> int:
        n = C.c_size_t()
        check(lib().hm_packed_size(self._h, C.byref(n)))
        return n.value

    def Pack(self) -> bytes:
        """The reference's byte layout of this H-matrix (Pack)."""
        n = self.PackedSize()
        buf = C.create_string_buffer(n)
        w = C.c_size_t()
        check(lib().hm_pack(self._h, buf, n, C.byref(w)))
        return buf.raw[:w.value]

    @classmethod
    def Unpack(cls, packed: bytes, ctx: Optional[Context] = None):
        """H-matrix from the reference's byte layout (the HMat2d(const
        Vector<byte>&) constructor)."""
        ctx = _ctx(ctx)
        buf = C.create_string_buffer(bytes(packed), len(packed))
        h = C.c_void_p()
        check(lib().hm_unpack(ctx.handle, cls.dim, buf, len(packed), C.byref(h)))
        return cls(ctx=ctx, _handle=h)

    def SetToRandom(self):
        """SetToRandom (src/HMat2d/SetToRandom-incl.hpp:14-55)."""
        check(lib().hm_set_to_random(self._h))

    # -- H * dense ------------------------------------------------------------
    def _apply_complex(self, op: int, alpha, B, beta, Cout):
        """Complex Multiply / TransposeMultiply / AdjointMultiply (op 0 / 1 /
        2) on host arrays through the engine's complex entry."""
        n = self.Height()
        Bn = np.asarray(B, dtype=np.complex128)
        vec = Bn.ndim == 1
        B2 = np.asfortranarray(Bn.reshape(-1, 1) if vec else Bn)
        if B2.shape[0] != n:
            raise _lib.HMError(1, "nonconformal multiply")
        k = B2.shape[1]
        if Cout is None:
            C2 = np.zeros((n, k), dtype=np.complex128, order="F")
        else:
            C2 = np.asfortranarray(np.asarray(Cout, dtype=np.complex128).reshape(n, k))
        a, b = complex(alpha), complex(beta)
        check(lib().hm_multiply_dense_complex_host(
            self._h, op, a.real, a.imag, B2.ctypes.data_as(_lib._PD), n, b.real, b.imag,
            C2.ctypes.data_as(_lib._PD), n, k))
        return C2[:, 0].copy() if vec else C2

    def _apply(self, transpose: int, alpha: float, B, beta: float, Cout):
        if self.is_complex:
            return self._apply_complex(transpose, alpha, B, beta, Cout)
        n = self.Height() if transpose else self.Width()
        m = self.Width() if transpose else self.Height()
        if _is_cuda_tensor(B):
            import torch
            vec = B.dim() == 1
            B2 = B.reshape(-1, 1) if vec else B
            if B2.dtype != torch.float64:
                raise _lib.HMError(1, "dense operands must be float64")
            # column-major view: a (n x k) column-major matrix is a k x n row-major tensor
            Bt = B2.t().contiguous() if not B2.t().is_contiguous() else B2.t()
            k = B2.shape[1]
            if B2.shape[0] != n:
                raise _lib.HMError(1, "nonconformal multiply")
            if Cout is None:
                Ct = torch.zeros((k, m), dtype=torch.float64, device=B.device)
            else:
                C2 = Cout.reshape(-1, 1) if Cout.dim() == 1 else Cout
                Ct = C2.t().contiguous()
            # the engine runs on its context's stream: order it after torch's
            # work on the operands, and torch's later reads after the product
            torch.cuda.current_stream(B.device).synchronize()
            check(lib().hm_multiply_dense(self._h, transpose, float(alpha), C.c_void_p(Bt.data_ptr()),
                                          n, float(beta), C.c_void_p(Ct.data_ptr()), m, k))
            self.ctx.synchronize()
            Cres = Ct.t()
            if Cout is not None:
                (Cout.reshape(-1, 1) if Cout.dim() == 1 else Cout).copy_(Cres)
                return Cout
            return Cres.reshape(-1) if vec else Cres
        Bn = np.asarray(B, dtype=np.float64)
        vec = Bn.ndim == 1
        B2 = np.asfortranarray(Bn.reshape(-1, 1) if vec else Bn)
        if B2.shape[0] != n:
            raise _lib.HMError(1, "nonconformal multiply")
        k = B2.shape[1]
        if Cout is None:
            C2 = np.zeros((m, k), order="F")
        else:
            C2 = np.asfortranarray(np.asarray(Cout, dtype=np.float64).reshape(m, k))
        check(lib().hm_multiply_dense_host(self._h, transpose, float(alpha),
                                           B2.ctypes.data_as(_lib._PD), n, float(beta),
                                           C2.ctypes.data_as(_lib._PD), m, k))
        return C2[:, 0].copy() if vec else C2

    def Multiply(self, alpha, B, beta=None, C=None):
        """Multiply (hmat2d.hpp:150-268).

        * ``Multiply(alpha, x)`` / ``Multiply(alpha, B)``: y = alpha H x for a
          vector or dense matrix (numpy array or CUDA float64 tensor);
        * ``Multiply(alpha, x, beta, y)``: y := alpha H x + beta y;
        * ``Multiply(alpha, B_hmat)`` / ``Multiply(alpha, B_hmat, beta, C)``:
          the H*H product with randomized compression.
        """
        if isinstance(B, _HMatBase):
            return self._multiply_hmat(alpha, B, beta, C)
        return self._apply(0, alpha, B, 0.0 if beta is None else beta, C)

    def TransposeMultiply(self, alpha, B, beta=None, C=None):
        """TransposeMultiply (hmat2d.hpp:162-206): C := alpha H^T B (+ beta C)."""
        return self._apply(1, alpha, B, 0.0 if beta is None else beta, C)

    def AdjointMultiply(self, alpha, B, beta=None, C=None):
        """AdjointMultiply: C := alpha H^H B (+ beta C); equal to
        TransposeMultiply for real scalars."""
        if self.is_complex:
            return self._apply_complex(2, alpha, B, 0.0 if beta is None else beta, C)
        return self.TransposeMultiply(alpha, B, beta, C)

    def _multiply_hmat(self, alpha, B, beta, Cm):
        """H*H (MultiplyHMat-incl.hpp:12-380).  Without beta: C = alpha A B,
        rebuilt (a new H-matrix unless C is given); with beta: C :~= alpha A B
        + beta C in place on C's structure."""
        if beta is None:
            out = _handle_of(Cm)
            check(lib().hm_multiply_hmat(self._h, float(alpha), B.handle, C.byref(out)))
            if Cm is not None:
                Cm._h = out
                return Cm
            return type(self)(ctx=self.ctx, _handle=out)
        if Cm is None or not Cm.handle:
            raise _lib.HMError(1, "C is required with beta")
        check(lib().hm_multiply_hmat_update(self._h, float(alpha), B.handle, float(beta),
                                            Cm.handle))
        return Cm

    # -- structural / elementwise (HMat2d.cpp:331-744) ---------------------
    def CopyFrom(self, B: "_HMatBase"):
        """A := B (CopyFrom, HMat2d.cpp:331-391)."""
        out = _handle_of(self)
        check(lib().hm_copy(B.handle, C.byref(out)))
        self._h = out
        return self

    def AdjointFrom(self, B: "_HMatBase"):
        """A := B^H (= B^T for real scalars; AdjointFrom, HMat2d.cpp:545-614)."""
        out = _handle_of(self)
        check(lib().hm_transpose(B.handle, C.byref(out)))
        self._h = out
        return self

    def TransposeFrom(self, B: "_HMatBase"):
        """A := B^T (TransposeFrom, HMat2d.cpp:477-546; B^T = B^H for real
        scalars, conj(B^H) for complex ones)."""
        if B.is_complex:
            out = _handle_of(self)
            check(lib().hm_transpose_complex(B.handle, C.byref(out)))
            self._h = out
            return self
        return self.AdjointFrom(B)

    def UpdateWith(self, alpha: float, B: "_HMatBase"):
        """A := alpha B + A (UpdateWith, HMat2d.cpp:749-781): low-rank blocks
        by RoundedUpdate to maxRank, dense blocks added."""
        check(lib().hm_update_with(self._h, float(alpha), B.handle))

    def SetToIdentity(self):
        """A := I (SetToIdentity, HMat2d.cpp:652-702): low-rank blocks emptied,
        dense diagonal I."""
        check(lib().hm_set_to_identity(self._h))

    def Conjugate(self):
        """A := conj(A) (Conjugate, HMat2d.cpp:396-422); nothing for real."""
        check(lib().hm_conjugate_in_place(self._h))

    def ConjugateFrom(self, B: "_HMatBase"):
        """A := conj(B) (ConjugateFrom, HMat2d.cpp:424-472); complex only."""
        out = _handle_of(self)
        check(lib().hm_conjugate(B.handle, C.byref(out)))
        self._h = out
        return self

    def Scale(self, alpha):
        """A := alpha A (HMat2d.cpp:616-647); complex alpha on complex matrices."""
        if isinstance(alpha, complex) or np.iscomplexobj(alpha):
            a = complex(alpha)
            check(lib().hm_scale_complex(self._h, a.real, a.imag))
        else:
            check(lib().hm_scale(self._h, float(alpha)))

    def AddConstantToDiagonal(self, alpha):
        """A := A + alpha I (HMat2d.cpp:704-744); complex alpha on complex matrices."""
        if isinstance(alpha, complex) or np.iscomplexobj(alpha):
            a = complex(alpha)
            check(lib().hm_add_constant_to_diagonal_complex(self._h, a.real, a.imag))
        else:
            check(lib().hm_add_constant_to_diagonal(self._h, float(alpha)))

    def DirectInvert(self):
        """A := inv(A) by recursive Schur complements
        (src/HMat2d/Invert-incl.hpp:17-125, src/HMat3d/Invert-incl.hpp:14-122)."""
        check(lib().hm_direct_invert(self._h))

    def SchulzInvert(self, numIterations: int, theta: float = 1.5, confidence: float = 6.0,
                     stopTol: float = 1e-4):
        """A :~= inv(A) by Schulz iteration (src/HMat2d/Invert-incl.hpp:127-196).

        Returns (iterations run, [estimate of ||A||, estimates of
        ||I - X_k A|| at each stop check])."""
        its = C.c_int()
        cap = 64
        trace = (C.c_double * cap)()
        n = C.c_int()
        check(lib().hm_schulz_invert(self._h, int(numIterations), float(theta),
                                     float(confidence), float(stopTol), C.byref(its), trace,
                                     cap, C.byref(n)))
        return its.value, [trace[i] for i in range(min(n.value, cap))]

    def SchulzInvertMixed(self, numIterations: int, theta: float = 1.5,
                          confidence: float = 6.0, stopTol: float = 1e-4,
                          mixedSwitch: float = 1e-2):
        """Mixed-precision SchulzInvert: iterations run their H*H products in
        the low-precision phase (TF32 range samples, FP32 roundings) while
        the last ||I - X_k A|| estimate is above mixedSwitch, then FP64.

        Returns (iterations run, low-precision iterations, trace)."""
        its, low = C.c_int(), C.c_int()
        cap = 64
        trace = (C.c_double * cap)()
        n = C.c_int()
        check(lib().hm_schulz_invert_mixed(self._h, int(numIterations), float(theta),
                                           float(confidence), float(stopTol), float(mixedSwitch),
                                           C.byref(its), C.byref(low), trace, cap, C.byref(n)))
        return its.value, low.value, [trace[i] for i in range(min(n.value, cap))]


def _handle_of(obj) -> C.c_void_p:
    """A fresh c_void_p holding obj's handle (NULL for None or an empty object)."""
    if obj is None or not obj.handle:
        return C.c_void_p(None)
    return C.c_void_p(obj.handle.value)


def EstimateTwoNorm(A: _HMatBase, theta: float, confidence: float) -> float:
    """hmat_tools::EstimateTwoNorm (include/dmhm/hmat_tools.hpp:1504-1548)."""
    v = C.c_double()
    check(lib().hm_estimate_two_norm(A.handle, float(theta), float(confidence), C.byref(v)))
    return v.value


class HMat2d(_HMatBase):
    """HMat2d<double> (include/dmhm/hmat2d.hpp:22-393)."""
    dim = 2

    def __init__(self, S: Optional[Sparse] = None, numLevels: int = 1, maxRank: int = 0,
                 stronglyAdmissible: bool = True, xSize: int = 0, ySize: int = 0,
                 ctx: Optional[Context] = None, _handle=None):
        super().__init__(S, numLevels, maxRank, stronglyAdmissible, xSize, ySize,
                         ctx=ctx, _handle=_handle)

    @staticmethod
    def BuildNaturalToHierarchicalMap(xSize: int, ySize: int, numLevels: int) -> np.ndarray:
        return natural_to_hierarchical_map((xSize, ySize), numLevels)


class HMat3d(_HMatBase):
    """HMat3d<double> (include/dmhm/hmat3d.hpp)."""
    dim = 3

    def __init__(self, S: Optional[Sparse] = None, numLevels: int = 1, maxRank: int = 0,
                 stronglyAdmissible: bool = True, xSize: int = 0, ySize: int = 0,
                 zSize: int = 0, ctx: Optional[Context] = None, _handle=None):
        super().__init__(S, numLevels, maxRank, stronglyAdmissible, xSize, ySize, zSize,
                         ctx=ctx, _handle=_handle)

    @staticmethod
    def BuildNaturalToHierarchicalMap(xSize: int, ySize: int, zSize: int,
                                      numLevels: int) -> np.ndarray:
        return natural_to_hierarchical_map((xSize, ySize, zSize), numLevels)


class _DistOps:
    """Single-rank DistHMat2d / DistHMat3d (include/dmhm/dist_hmat2d.hpp): the
    whole matrix is local, products truncate by the global
    CompressionTolerance (SVDTrunc, src/DistHMat2d/Truncation-incl.hpp:37-63),
    and multType has no effect on the result.  The reference compresses with
    two-sided sketches and Gram eigendecompositions; this engine rounds with
    QR and a Jacobi SVD under the same truncation rule, so results agree to
    the tolerance's scale."""

    def LocalHeight(self) -> int:
        return self.Height()

    def LocalWidth(self) -> int:
        return self.Width()

    def FirstLocalRow(self) -> int:
        return 0

    def FirstLocalCol(self) -> int:
        return 0

    def ParallelEstimateTwoNorm(self, theta: float, confidence: float) -> float:
        """ParallelEstimateTwoNorm (src/DistHMat2d/Norm-incl.hpp:12-77)."""
        return EstimateTwoNorm(self, theta, confidence)

    def Multiply(self, alpha, B, beta=None, C=None, multType: int = 2):
        """Vectors and dense blocks as HMat2d; H*H C := alpha A B under the
        global compression tolerance (MultiplyHMat-incl.hpp:28-52)."""
        if isinstance(B, _HMatBase):
            with _ScopedTolerance(self.ctx, CompressionTolerance()):
                return super().Multiply(alpha, B, beta, C)
        return super().Multiply(alpha, B, beta, C)

    def SchulzInvert(self, numIterations: int, multType: int = 2, theta: float = 1.5,
                     confidence: float = 6.0, stopTol: float = 1e-4, printRank: bool = False):
        """SchulzInvert (src/DistHMat2d/Invert-incl.hpp:14-105) under the global
        compression tolerance."""
        with _ScopedTolerance(self.ctx, CompressionTolerance()):
            return super().SchulzInvert(numIterations, theta, confidence, stopTol)


class Teams:
    """Teams(mpi::Comm) of the distributed classes: one team of one process."""

    def __init__(self, comm=None):
        self.comm = comm

    def NumLevels(self) -> int:
        return 1


class DistHMat2d(_DistOps, HMat2d):
    """Single-rank DistHMat2d<double> (include/dmhm/dist_hmat2d.hpp)."""

    def __init__(self, S: Optional[Sparse] = None, numLevels: int = 1, maxRank: int = 0,
                 stronglyAdmissible: bool = True, xSize: int = 0, ySize: int = 0,
                 teams: Optional[Teams] = None, ctx: Optional[Context] = None, _handle=None):
        HMat2d.__init__(self, S, numLevels, maxRank, stronglyAdmissible, xSize, ySize,
                        ctx=ctx, _handle=_handle)


class DistHMat3d(_DistOps, HMat3d):
    """Single-rank DistHMat3d<double> (include/dmhm/dist_hmat3d.hpp)."""

    def __init__(self, S: Optional[Sparse] = None, numLevels: int = 1, maxRank: int = 0,
                 stronglyAdmissible: bool = True, xSize: int = 0, ySize: int = 0,
                 zSize: int = 0, teams: Optional[Teams] = None, ctx: Optional[Context] = None,
                 _handle=None):
        HMat3d.__init__(self, S, numLevels, maxRank, stronglyAdmissible, xSize, ySize, zSize,
                        ctx=ctx, _handle=_handle)


class RankModel:
    """Learned rank predictor of the randomized H*H compressions (a 3-layer
    perceptron trained and evaluated by the library's GPU kernels)."""

    def __init__(self, ctx: Optional[Context] = None, seed: int = 1):
        self.ctx = _ctx(ctx)
        h = C.c_void_p()
        check(lib().hm_rank_model_create(self.ctx.handle, C.c_uint64(seed), C.byref(h)))
        self._h = h

    @property
    def handle(self):
        return self._h

    @staticmethod
    def num_features() -> int:
        return lib().hm_rank_feature_count()

    @staticmethod
    def num_params() -> int:
        return lib().hm_rank_param_count()

    def close(self):
        if self._h:
            lib().hm_rank_model_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _f32(a):
        import numpy as np
        return np.ascontiguousarray(a, dtype=np.float32)

    def params(self):
        import numpy as np
        p = np.zeros(self.num_params(), dtype=np.float32)
        check(lib().hm_rank_model_get_params(self._h, p.ctypes.data_as(C.POINTER(C.c_float)), p.size))
        return p

    def set_params(self, p):
        p = self._f32(p)
        check(lib().hm_rank_model_set_params(self._h, p.ctypes.data_as(C.POINTER(C.c_float)), p.size))

    def loss_grad(self, x, t):
        import numpy as np
        x, t = self._f32(x), self._f32(t)
        g = np.zeros(self.num_params(), dtype=np.float32)
        loss = C.c_float()
        P = C.POINTER(C.c_float)
        check(lib().hm_rank_model_loss_grad(self._h, x.ctypes.data_as(P), t.ctypes.data_as(P),
                                            t.size, C.byref(loss), g.ctypes.data_as(P)))
        return float(loss.value), g

    def train(self, x, t, epochs: int = 500, lr: float = 1e-2) -> float:
        x, t = self._f32(x), self._f32(t)
        loss = C.c_float()
        P = C.POINTER(C.c_float)
        check(lib().hm_rank_model_train(self._h, x.ctypes.data_as(P), t.ctypes.data_as(P), t.size,
                                        int(epochs), C.c_float(lr), C.byref(loss)))
        return float(loss.value)

    def predict(self, x):
        import numpy as np
        x = self._f32(x)
        n = x.shape[0]
        out = np.zeros(n, dtype=np.float32)
        P = C.POINTER(C.c_float)
        check(lib().hm_rank_model_predict(self._h, x.ctypes.data_as(P), n, out.ctypes.data_as(P)))
        return out
