"""Oracle of Fortran's RESHAPE(SOURCE, SHAPE, ORDER=order) for pure
transposes (test infrastructure only): the source is read in array element
order and the result filled with its subscripts running in the order
order(1), order(2), ...; the redistribution transposes of
src/green_rgf.f90:243-329 are of this form."""
import numpy as np


def fortran_reshape_order(flat, src_shape, order):
    """flat: 1-D array (column-major data of src_shape); order 1-based."""
    src = np.asarray(flat).reshape(src_shape, order="F")
    nd = len(src_shape)
    axes = [0] * nd                      # destination axis j takes source axis axes[j]
    for k in range(nd):
        axes[order[k] - 1] = k
    return src.transpose(axes).reshape(-1, order="F")


def fortran_reshape_order_loops(flat, src_shape, order):
    """The same by the intrinsic's definition, element by element (small)."""
    nd = len(src_shape)
    dst_shape = [0] * nd
    for k in range(nd):
        dst_shape[order[k] - 1] = src_shape[k]
    out = np.empty(int(np.prod(src_shape)), dtype=np.asarray(flat).dtype)
    idx = [0] * nd                       # destination subscripts, run in the order `order`
    for p in range(out.size):
        lin, mult = 0, 1
        for d in range(nd):
            lin += idx[d] * mult
            mult *= dst_shape[d]
        out[lin] = flat[p]
        for k in range(nd):              # next subscript tuple in ORDER sequence
            d = order[k] - 1
            idx[d] += 1
            if idx[d] < dst_shape[d]:
                break
            idx[d] = 0
    return out
