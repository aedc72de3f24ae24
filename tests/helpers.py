"""Shared test helpers: golden-case decoding and the reference's comparisons."""
import numpy as np

import oracle as O

BORDER_NAMES = {O.ZERO: "BorderZero", O.CLAMP: "BorderClamp", O.CYCLIC: "BorderCyclic",
                O.VALID: "BorderValid", O.FULL: "BorderFull"}
# Adjoint border of each forward border (Valid <-> Full); Clamp has none.
ADJOINT_BORDER = {O.ZERO: O.ZERO, O.CYCLIC: O.CYCLIC, O.VALID: O.FULL, O.FULL: O.VALID}
ADJOINT_SAMPLING = {O.NOSAMPLE: O.NOSAMPLE, O.DOWN: O.UP, O.UP: O.DOWN}


def golden_case(golden, i):
    sampling, step, border = (int(v) for v in golden[f"hdr{i}"])
    arrays = {n: golden[f"{n}{i}"] for n in ("x", "k", "wx", "y", "wty")}
    return sampling, step, border, arrays


def legal_in_reference(sampling, step, border):
    """DynamicConvolutionSpec.scala:157-160 skips Upsample+Clamp, which
    DynamicConvolutionGenerator.scala:530-535 rejects."""
    return not (sampling == O.UP and step > 1 and border == O.CLAMP)


def ref_field_approx_equal(a, b):
    """RefFieldMemory.~== (src/test/scala/cogx/reference/memory/RefFieldMemory.scala:433-485):
    each element within 0.001 absolute, or within 1e-5 relative."""
    a = np.asarray(a, dtype=np.float32)
    b = np.asarray(b, dtype=np.float32)
    if a.shape != b.shape:
        return False
    diff = np.abs(a - b)
    close = diff <= 0.001
    with np.errstate(divide="ignore", invalid="ignore"):
        rel = np.abs(a / b - 1.0)
    rel_ok = (b != 0) & (rel <= 1e-5)
    return bool(np.all(close | rel_ok))


def bitwise_equal(a, b):
    a = np.asarray(a, dtype=np.float32)
    b = np.asarray(b, dtype=np.float32)
    return a.shape == b.shape and bool(np.all((a == b) | (np.isnan(a) & np.isnan(b))))
