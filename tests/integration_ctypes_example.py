import ctypes, numpy as np
L = ctypes.CDLL("parallel-ra_b200/libra_b200.so")
P = ctypes.c_void_p; I = ctypes.POINTER(ctypes.c_int); U = ctypes.POINTER(ctypes.c_uint64)
L.ra_program_create.argtypes = [ctypes.c_int, ctypes.POINTER(P)]
L.ra_relation_create.argtypes = [P, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_char_p, ctypes.c_int, I]
L.ra_relation_load_rows.argtypes = [P, ctypes.c_int, U, ctypes.c_uint64]
L.ra_scc_create.argtypes = [P, ctypes.c_int, ctypes.c_int, I]
L.ra_scc_add_relation.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_int]
L.ra_scc_add_join.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, I, ctypes.c_int]
L.ra_scc_add_copy.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, I, ctypes.c_int, ctypes.c_int]
L.ra_scc_depend.argtypes = [P, ctypes.c_int, ctypes.c_int]
L.ra_program_execute.argtypes = [P]
L.ra_relation_counts.argtypes = [P, ctypes.c_int, U, U]

p = P(); L.ra_program_create(0, ctypes.byref(p))
T, G = ctypes.c_int(), ctypes.c_int()
L.ra_relation_create(p, 1, 2, 257, b"T", 1, ctypes.byref(T))
L.ra_relation_create(p, 1, 2, 256, b"G", 1, ctypes.byref(G))
edges = np.array([[0, 1, 0], [1, 2, 1]], dtype=np.uint64)          # (src, dst, id)
L.ra_relation_load_rows(p, G, edges.ctypes.data_as(U), len(edges))
join, copy = ctypes.c_int(), ctypes.c_int()
L.ra_scc_create(p, 1, 1, ctypes.byref(join)); L.ra_scc_create(p, 0, 2, ctypes.byref(copy))
for s, init in ((join, 1), (copy, 1)):
    L.ra_scc_add_relation(p, s, G, 0); L.ra_scc_add_relation(p, s, T, init)
L.ra_scc_add_join(p, join, T, T, 0, G, 1, (ctypes.c_int * 2)(3, 1), 2)   # T(z,x) :- T(y,x), G(y,z)
L.ra_scc_add_copy(p, copy, 0, T, G, 1, (ctypes.c_int * 2)(1, 0), 2, 0)   # T(y,x) :- G(x,y)
L.ra_scc_depend(p, copy, join)
L.ra_program_execute(p)
f, d = ctypes.c_uint64(), ctypes.c_uint64()
L.ra_relation_counts(p, T, ctypes.byref(f), ctypes.byref(d))      # f.value == 3
