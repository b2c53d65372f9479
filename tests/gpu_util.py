"""Helpers shared by the GPU tests: device tree export through the C ABI."""
import ctypes as C

import numpy as np


def device_tree(src, trg, idivflag, ndiv, nlmax=51):
    import torch
    from fmm2d_b200 import _lib
    L = _lib.lib()
    s = torch.as_tensor(np.ascontiguousarray(src.T)).cuda()
    ns = src.shape[1]
    if trg is None:
        t, nt = None, 0
    else:
        t = torch.as_tensor(np.ascontiguousarray(trg.T)).cuda()
        nt = trg.shape[1]
    nl, nb, ier = C.c_int(), C.c_int(), C.c_int()
    h = L.b2fmm_tree_build(C.c_void_p(s.data_ptr()), ns, C.c_void_p(t.data_ptr() if t is not None else None),
                           nt, idivflag, ndiv, nlmax, C.byref(nl), C.byref(nb), C.byref(ier))
    assert ier.value == 0, ier.value
    nl, nb = nl.value, nb.value
    i32 = lambda *shape: np.zeros(shape, dtype=np.int32)
    out = dict(nlevels=nl, nboxes=nb, laddr=i32(nl + 1, 2), ilevel=i32(nb), iparent=i32(nb),
               nchild=i32(nb), ichild=i32(nb, 4), ncoll=i32(nb), coll=i32(nb, 9),
               centers=np.zeros((nb, 2)), boxsize=np.zeros(nl + 1), isrc=i32(ns),
               isrcse=i32(nb, 2), itarg=i32(nt), itargse=i32(nb, 2), nlist1=i32(nb),
               list1=i32(nb, 13), nlist2=i32(nb), list2=i32(nb, 27), nlist3=i32(nb),
               list3=i32(nb, 20), nlist4=i32(nb), list4=i32(nb, 5))
    keys = ["laddr", "ilevel", "iparent", "nchild", "ichild", "ncoll", "coll", "centers",
            "boxsize", "isrc", "isrcse", "itarg", "itargse", "nlist1", "list1", "nlist2", "list2",
            "nlist3", "list3", "nlist4", "list4"]
    L.b2fmm_tree_get(C.c_void_p(h), *[out[k].ctypes.data_as(C.c_void_p) for k in keys],
                     C.byref(ier))
    assert ier.value == 0
    L.b2fmm_tree_free(C.c_void_p(h))
    return out
