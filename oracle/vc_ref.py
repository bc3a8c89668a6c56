"""Test infrastructure: a CPU restatement of the reference's volume-control
truncation, mod_3dbem_system_vc (src/Solvers/system_assembly.cpp:560-629),
in plain Python loops over element nodes, the checker of
hfpx_matrix_truncate and of the host right-hand-side gather.  It is not used
by the product.

The loops follow the reference: for every element node (s_ele, j) kept by
the truncated handle (dof_h >= 0) and every kept (t_ele, k), matrix(t, s)
+= orig(o_t, o_s); the volume row and pressure column of s; and the
right-hand side chosen by the length of delta_t (the full element-node
numbering, the original DoF numbering, or the truncated one).  The one
change: the reference reads the border at row and column full_ndof of a
matrix it first requires to be orig_ndof square (system_assembly.cpp:575,
607-611), one past its end; here orig is the bordered matrix
(make_3dbem_matrix_vc, :458-557) and its border is its own last row and
column.  The corner stays 0 as in the reference, which never writes it.

Parity: unpinned against the reference itself, whose function cannot run
as written (the read past the end); pinned on the reference's own loop
structure restated here and on numpy index gathers in the tests.
"""
import numpy as np


def mod_3dbem_system_vc(orig, orig_dof_h, dof_h, delta_t, delta_v):
    """orig: bordered matrix (orig_ndof + 1 square); orig_dof_h, dof_h: n_el x
    18 DoF handles (-1 fixed) -> (matrix (used + 1 square), rhs (used + 1))."""
    orig = np.asarray(orig, dtype=np.float64)
    od = np.asarray(orig_dof_h, dtype=np.int64)
    td = np.asarray(dof_h, dtype=np.int64)
    n_el, ndpe = od.shape
    full = n_el * ndpe
    orig_ndof = orig.shape[0] - 1
    border = orig_ndof
    used = int(td.max()) + 1
    dt = np.asarray(delta_t, dtype=np.float64).reshape(-1)
    assert dt.size in (full, orig_ndof, used)
    mat = np.zeros((used + 1, used + 1))
    rhs = np.zeros(used + 1)
    rhs[used] = delta_v
    for s_ele in range(n_el):
        for j in range(ndpe):
            s = int(td[s_ele, j])
            if s < 0:
                continue
            o_s = int(od[s_ele, j])
            for t_ele in range(n_el):
                for k in range(ndpe):
                    t = int(td[t_ele, k])
                    if t >= 0:
                        mat[t, s] += orig[int(od[t_ele, k]), o_s]
            mat[used, s] += orig[border, o_s]
            mat[s, used] += orig[o_s, border]
            if dt.size == full:
                rhs[s] = dt[s_ele * ndpe + j]
            elif dt.size == orig_ndof:
                rhs[s] = dt[o_s]
            else:
                rhs[s] = dt[s]
    return mat, rhs


def truncate_handle(orig_dof_h, drop):
    """A truncated handle as the reference's contact iteration makes one
    (src/Development/c_f_iteration.cpp:212-258): walking the element nodes in
    order, a dropped DoF becomes -1 and every later kept DoF moves down by
    the number dropped so far.  drop: boolean n_el x 18."""
    od = np.asarray(orig_dof_h, dtype=np.int64)
    out = np.full(od.shape, -1, dtype=np.int64)
    dec = 0
    n_el, ndpe = od.shape
    for el in range(n_el):
        for j in range(ndpe):
            if od[el, j] < 0:
                continue
            if drop[el, j]:
                dec += 1
            else:
                out[el, j] = od[el, j] - dec
    return out
