"""ctypes binding of the libCEED API subset exported by libceed_b200.so.

Object names and call sequences follow libCEED as HONEE uses it (src/setuplibceed.c, src/qdata.c, src/setupts.c,
src/mat-ceed.c), so Python code written against this module reads like the reference's C.  Every call checks the
returned error code and raises :class:`CeedError` with the message stored by CeedErrorStore (examples/navierstokes.c:66,
include/petsc-ceed.h:25-36 wrap every call the same way).
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import lib as _load

CEED_MEM_HOST, CEED_MEM_DEVICE = 0, 1
CEED_COPY_VALUES, CEED_USE_POINTER, CEED_OWN_POINTER = 0, 1, 2
CEED_NORM_1, CEED_NORM_2, CEED_NORM_MAX = 0, 1, 2
CEED_NOTRANSPOSE, CEED_TRANSPOSE = 0, 1
CEED_EVAL_NONE, CEED_EVAL_INTERP, CEED_EVAL_GRAD, CEED_EVAL_WEIGHT = 0, 1, 2, 16
CEED_GAUSS, CEED_GAUSS_LOBATTO = 0, 1
CEED_ERROR_SUCCESS, CEED_ERROR_UNSUPPORTED = 0, -3

_vp = C.c_void_p
_dp = C.POINTER(C.c_double)


class CeedError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"libCEED error {code}: {msg}")
        self.code = code


def L():
    return _load()


def _sym(name):
    return C.c_void_p.in_dll(L(), name).value


def _chk(ceed_ptr, code):
    if code != 0:
        msg = C.c_char_p()
        L().CeedGetErrorMessage(_vp(ceed_ptr), C.byref(msg))
        raise CeedError(code, (msg.value or b"").decode(errors="replace"))


class Ceed:
    """CeedInit(resource) (examples/navierstokes.c:64)."""

    def __init__(self, resource: str = "/gpu/b200"):
        self.ptr = _vp()
        code = L().CeedInit(resource.encode(), C.byref(self.ptr))
        if code:
            _chk(None, code)
        self.resource = resource

    def chk(self, code):
        _chk(self.ptr.value, code)

    def destroy(self):
        if self.ptr.value:
            L().CeedDestroy(C.byref(self.ptr))

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    @property
    def active(self):
        return _vp(_sym("CEED_VECTOR_ACTIVE"))

    @property
    def vector_none(self):
        return _vp(_sym("CEED_VECTOR_NONE"))

    @property
    def basis_none(self):
        return _vp(_sym("CEED_BASIS_NONE"))

    @property
    def rstr_none(self):
        return _vp(_sym("CEED_ELEMRESTRICTION_NONE"))

    @property
    def strides_backend(self):
        return C.cast(C.c_void_p(C.addressof(C.c_int32.in_dll(L(), "CEED_STRIDES_BACKEND"))), C.POINTER(C.c_int32))

    @property
    def request_immediate(self):
        return _vp(_sym("CEED_REQUEST_IMMEDIATE"))


class _Obj:
    _destroy = None

    def __init__(self, ceed: Ceed):
        self.ceed = ceed
        self.ptr = _vp()

    def destroy(self):
        if self.ptr.value and self._destroy:
            getattr(L(), self._destroy)(C.byref(self.ptr))

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


class Vector(_Obj):
    _destroy = "CeedVectorDestroy"

    def __init__(self, ceed: Ceed, length: int):
        super().__init__(ceed)
        ceed.chk(L().CeedVectorCreate(ceed.ptr, C.c_ssize_t(length), C.byref(self.ptr)))
        self.length = length
        self._keep = None

    @classmethod
    def wrap(cls, ceed, ptr, length):
        v = cls.__new__(cls)
        _Obj.__init__(v, ceed)
        v.ptr = _vp(ptr)
        v.length = length
        v._keep = None
        return v

    def set_array_host(self, arr: np.ndarray, copy: bool = True):
        arr = np.ascontiguousarray(arr, dtype=np.float64)
        assert arr.size == self.length
        self._keep = None if copy else arr
        self.ceed.chk(L().CeedVectorSetArray(self.ptr, CEED_MEM_HOST, CEED_COPY_VALUES if copy else CEED_USE_POINTER, arr.ctypes.data_as(_dp)))

    def set_array_device(self, dev_ptr: int, copy: bool = False, keep=None):
        """Wrap (CEED_USE_POINTER) or copy a device array, e.g. torch_tensor.data_ptr() (include/petsc-ceed-utils.h:127-191)."""
        self._keep = keep
        self.ceed.chk(L().CeedVectorSetArray(self.ptr, CEED_MEM_DEVICE, CEED_COPY_VALUES if copy else CEED_USE_POINTER, C.cast(_vp(dev_ptr), _dp)))

    def take_array_device(self) -> int:
        p = _dp()
        self.ceed.chk(L().CeedVectorTakeArray(self.ptr, CEED_MEM_DEVICE, C.byref(p)))
        self._keep = None
        return C.cast(p, _vp).value or 0

    def set_value(self, v: float):
        self.ceed.chk(L().CeedVectorSetValue(self.ptr, C.c_double(v)))

    def to_numpy(self) -> np.ndarray:
        p = _dp()
        self.ceed.chk(L().CeedVectorGetArrayRead(self.ptr, CEED_MEM_HOST, C.byref(p)))
        out = np.ctypeslib.as_array(p, shape=(self.length,)).copy()
        self.ceed.chk(L().CeedVectorRestoreArrayRead(self.ptr, C.byref(p)))
        return out

    def device_ptr(self, write=False) -> int:
        p = _dp()
        fn = L().CeedVectorGetArray if write else L().CeedVectorGetArrayRead
        self.ceed.chk(fn(self.ptr, CEED_MEM_DEVICE, C.byref(p)))
        addr = C.cast(p, _vp).value
        (L().CeedVectorRestoreArray if write else L().CeedVectorRestoreArrayRead)(self.ptr, C.byref(p))
        return addr

    def norm(self, kind=CEED_NORM_2) -> float:
        r = C.c_double()
        self.ceed.chk(L().CeedVectorNorm(self.ptr, kind, C.byref(r)))
        return r.value

    def axpy(self, alpha, x: "Vector"):
        self.ceed.chk(L().CeedVectorAXPY(self.ptr, C.c_double(alpha), x.ptr))

    def scale(self, alpha):
        self.ceed.chk(L().CeedVectorScale(self.ptr, C.c_double(alpha)))

    def copy_to(self, other: "Vector"):
        self.ceed.chk(L().CeedVectorCopy(self.ptr, other.ptr))

    def pointwise_mult(self, x: "Vector", y: "Vector"):
        self.ceed.chk(L().CeedVectorPointwiseMult(self.ptr, x.ptr, y.ptr))

    def reciprocal(self):
        self.ceed.chk(L().CeedVectorReciprocal(self.ptr))


class ElemRestriction(_Obj):
    _destroy = "CeedElemRestrictionDestroy"

    def __init__(self, ceed: Ceed, num_elem, elem_size, num_comp, comp_stride, l_size, offsets: Optional[np.ndarray] = None,
                 strides=None):
        super().__init__(ceed)
        self.num_elem, self.elem_size, self.num_comp, self.l_size = num_elem, elem_size, num_comp, l_size
        if offsets is not None:
            off = np.ascontiguousarray(offsets, dtype=np.int32)
            ceed.chk(L().CeedElemRestrictionCreate(ceed.ptr, num_elem, elem_size, num_comp, comp_stride, C.c_ssize_t(l_size), CEED_MEM_HOST,
                                                   CEED_COPY_VALUES, off.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(self.ptr)))
        else:
            if strides is None:
                sp = ceed.strides_backend
            else:
                arr = (C.c_int32 * 3)(*strides)
                sp = C.cast(arr, C.POINTER(C.c_int32))
            ceed.chk(L().CeedElemRestrictionCreateStrided(ceed.ptr, num_elem, elem_size, num_comp, C.c_ssize_t(l_size), sp, C.byref(self.ptr)))

    def create_vectors(self):
        lv, ev = _vp(), _vp()
        self.ceed.chk(L().CeedElemRestrictionCreateVector(self.ptr, C.byref(lv), C.byref(ev)))
        n_e = self.num_elem * self.elem_size * self.num_comp
        return Vector.wrap(self.ceed, lv.value, self.l_size), Vector.wrap(self.ceed, ev.value, n_e)

    def multiplicity(self, mult: Vector):
        """CeedElemRestrictionGetMultiplicity: mult = the number of element nodes at each L-vector entry."""
        self.ceed.chk(L().CeedElemRestrictionGetMultiplicity(self.ptr, mult.ptr))

    def apply(self, transpose: bool, u: Vector, ru: Vector):
        self.ceed.chk(L().CeedElemRestrictionApply(self.ptr, CEED_TRANSPOSE if transpose else CEED_NOTRANSPOSE, u.ptr, ru.ptr,
                                                   self.ceed.request_immediate))


class Basis(_Obj):
    _destroy = "CeedBasisDestroy"

    def __init__(self, ceed: Ceed, dim, num_comp, P, Q, interp1d=None, grad1d=None, qref1d=None, qweight1d=None, lagrange_mode=None):
        super().__init__(ceed)
        self.dim, self.num_comp, self.P, self.Q = dim, num_comp, P, Q
        if lagrange_mode is not None:
            ceed.chk(L().CeedBasisCreateTensorH1Lagrange(ceed.ptr, dim, num_comp, P, Q, lagrange_mode, C.byref(self.ptr)))
            return
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (interp1d, grad1d, qref1d, qweight1d)]
        ceed.chk(L().CeedBasisCreateTensorH1(ceed.ptr, dim, num_comp, P, Q, *[a.ctypes.data_as(_dp) for a in arrs], C.byref(self.ptr)))

    @classmethod
    def projection(cls, basis_from: "Basis", basis_to: "Basis"):
        """CeedBasisCreateProjection(basis_from, basis_to): interpolation from one basis's nodes onto the other's."""
        b = cls.__new__(cls)
        _Obj.__init__(b, basis_from.ceed)
        b.dim, b.num_comp, b.P, b.Q = basis_from.dim, basis_from.num_comp, basis_from.P, basis_to.P
        basis_from.ceed.chk(L().CeedBasisCreateProjection(basis_from.ptr, basis_to.ptr, C.byref(b.ptr)))
        return b

    def apply(self, num_elem, transpose, emode, u: Optional[Vector], v: Vector):
        self.ceed.chk(L().CeedBasisApply(self.ptr, num_elem, CEED_TRANSPOSE if transpose else CEED_NOTRANSPOSE, emode,
                                         u.ptr if u is not None else self.ceed.vector_none, v.ptr))


class QFunctionContext(_Obj):
    _destroy = "CeedQFunctionContextDestroy"

    def __init__(self, ceed: Ceed, struct_obj):
        """Wraps a ctypes Structure zero-copy (CEED_USE_POINTER, problems/newtonian.c:745); keep `struct_obj` alive."""
        super().__init__(ceed)
        ceed.chk(L().CeedQFunctionContextCreate(ceed.ptr, C.byref(self.ptr)))
        self.data = struct_obj
        ceed.chk(L().CeedQFunctionContextSetData(self.ptr, CEED_MEM_HOST, CEED_USE_POINTER, C.c_size_t(C.sizeof(struct_obj)),
                                                 C.cast(C.pointer(struct_obj), _vp)))

    def register_double(self, name: str, offset: int, num_values: int = 1, description: str = ""):
        self.ceed.chk(L().CeedQFunctionContextRegisterDouble(self.ptr, name.encode(), C.c_size_t(offset), C.c_size_t(num_values),
                                                             description.encode()))


class QFunction(_Obj):
    _destroy = "CeedQFunctionDestroy"

    def __init__(self, ceed: Ceed, source: str, vlength: int = 1):
        """CeedQFunctionCreateInterior(ceed, 1, f, f_loc, &qf); the backend binds by the kernel name in `source`."""
        super().__init__(ceed)
        ceed.chk(L().CeedQFunctionCreateInterior(ceed.ptr, vlength, None, source.encode(), C.byref(self.ptr)))

    def add_input(self, name, size, emode):
        self.ceed.chk(L().CeedQFunctionAddInput(self.ptr, name.encode(), size, emode))

    def add_output(self, name, size, emode):
        self.ceed.chk(L().CeedQFunctionAddOutput(self.ptr, name.encode(), size, emode))

    def set_context(self, ctx: QFunctionContext):
        self.ceed.chk(L().CeedQFunctionSetContext(self.ptr, ctx.ptr))


class Operator(_Obj):
    _destroy = "CeedOperatorDestroy"

    def __init__(self, ceed: Ceed, qf: Optional[QFunction] = None):
        super().__init__(ceed)
        if qf is None:
            ceed.chk(L().CeedOperatorCreateComposite(ceed.ptr, C.byref(self.ptr)))
        else:
            ceed.chk(L().CeedOperatorCreate(ceed.ptr, qf.ptr, None, None, C.byref(self.ptr)))
        self._subs = []

    def set_field(self, name, rstr, basis, vec):
        r = rstr.ptr if isinstance(rstr, ElemRestriction) else rstr
        b = basis.ptr if isinstance(basis, Basis) else basis
        v = vec.ptr if isinstance(vec, Vector) else vec
        self.ceed.chk(L().CeedOperatorSetField(self.ptr, name.encode(), r, b, v))

    def add_sub(self, sub: "Operator"):
        self.ceed.chk(L().CeedOperatorCompositeAddSub(self.ptr, sub.ptr))
        self._subs.append(sub)

    def set_name(self, name):
        self.ceed.chk(L().CeedOperatorSetName(self.ptr, name.encode()))

    def apply(self, inp: Optional[Vector], out: Optional[Vector], add=False):
        fn = L().CeedOperatorApplyAdd if add else L().CeedOperatorApply
        self.ceed.chk(fn(self.ptr, inp.ptr if inp is not None else self.ceed.vector_none,
                         out.ptr if out is not None else self.ceed.vector_none, self.ceed.request_immediate))

    def assemble_diagonal(self, out: Vector):
        self.ceed.chk(L().CeedOperatorLinearAssembleDiagonal(self.ptr, out.ptr, self.ceed.request_immediate))

    def assemble_point_block_diagonal(self, out: Vector):
        self.ceed.chk(L().CeedOperatorLinearAssemblePointBlockDiagonal(self.ptr, out.ptr, self.ceed.request_immediate))

    def point_block_symbolic(self):
        """(rows, cols) of CeedOperatorLinearAssemblePointBlockDiagonalSymbolic as numpy arrays (the C arrays are freed)."""
        n = C.c_int64()
        rows, cols = C.POINTER(C.c_int32)(), C.POINTER(C.c_int32)()
        self.ceed.chk(L().CeedOperatorLinearAssemblePointBlockDiagonalSymbolic(self.ptr, C.byref(n), C.byref(rows), C.byref(cols)))
        r = np.ctypeslib.as_array(rows, shape=(n.value,)).copy()
        c = np.ctypeslib.as_array(cols, shape=(n.value,)).copy()
        libc = C.CDLL(None)
        libc.free(C.cast(rows, C.c_void_p))
        libc.free(C.cast(cols, C.c_void_p))
        return r, c

    def context_label(self, name):
        lab = _vp()
        self.ceed.chk(L().CeedOperatorGetContextFieldLabel(self.ptr, name.encode(), C.byref(lab)))
        return lab

    def set_context_double(self, name, values):
        lab = self.context_label(name)
        if not lab.value:
            raise CeedError(-1, f"no context field '{name}'")
        vals = (C.c_double * len(values))(*values)
        self.ceed.chk(L().CeedOperatorSetContextDouble(self.ptr, lab, vals))

    def get_context_double(self, name):
        lab = self.context_label(name)
        n = C.c_size_t()
        p = _dp()
        self.ceed.chk(L().CeedOperatorGetContextDoubleRead(self.ptr, lab, C.byref(n), C.byref(p)))
        vals = [p[i] for i in range(n.value)]
        L().CeedOperatorRestoreContextDoubleRead(self.ptr, lab, C.byref(p))
        return vals

    def active_lengths(self):
        a, b = C.c_ssize_t(), C.c_ssize_t()
        self.ceed.chk(L().CeedOperatorGetActiveVectorLengths(self.ptr, C.byref(a), C.byref(b)))
        return a.value, b.value

    def flops(self):
        f = C.c_ssize_t()
        self.ceed.chk(L().CeedOperatorGetFlopsEstimate(self.ptr, C.byref(f)))
        return f.value
