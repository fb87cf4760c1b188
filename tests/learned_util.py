"""Shared helpers of the learned-preconditioner tests: the oracle's graph
tables for a plan (from the plan's exported leaf lists, neighbour lists and
RWGs, and the mesh)."""
import numpy as np


def oracle_graph(op, mesh, eps_r):
    from oracle import learned_precond as LP
    ptr, rwg = op.leaf_rwgs()
    ll = op.level_lists(op.max_level)
    rw = op.rwgs()
    pos = {int(f): i for i, f in enumerate(mesh.face_ids)}
    fp = np.array([pos[int(f)] for f in rw["face_pos"]])
    fn = np.array([pos[int(f)] for f in rw["face_neg"]])
    return LP.Graph(ptr, rwg, ll["near_ptr"], ll["near_idx"], mesh.points, mesh.faces, fp, fn, rw["length"], eps_r)
