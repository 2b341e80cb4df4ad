"""The property the short-list near-membrane kernels rest on, checked on the
oracle (bit for bit the reference's reflectionFed, Src/solfuncs.cpp:400-598):
a particle outside the periodic stencil bands none of whose list entries
passes the crossing test on the triangle's normals at t and t + dtmd
(bt * bdt <= 0 with the inside/outside flag clear) leaves the loop with its
state unchanged and a contact time of 0.  The first launch finishes exactly
those particles with free flight and walls; every other particle goes to the
queue, whose walk is the loop itself.  The test also bounds how many
particles need the queue, which is what makes the split pay."""
import ctypes as C

import numpy as np

import oracle as O


def _cp(a, b):
    # the reference's cross product (Src/memfuncs.cpp:96-108), operand order kept
    return np.stack([(a[:, 1] * b[:, 2]) - (b[:, 1] * a[:, 2]),
                     (a[:, 2] * b[:, 0]) - (b[:, 2] * a[:, 0]),
                     (a[:, 0] * b[:, 1]) - (b[:, 0] * a[:, 1])], 1)


def test_particles_without_a_crossing_candidate_leave_reflection_unchanged():
    Lx, Ly, Lz = 48.0, 32.0, 32.0
    p = O.default_params(Lx=Lx, Ly=Ly, Lz=Lz, Ns=int(Lx * Ly * (Lz + 1) * 10))
    orc = O.Oracle(p, 11)
    V, E, T = O.load_mesh_files(*O.troph_files())
    orc.init(V, E, T, 300)
    orc.step(11)  # past the first collision (step 10), with a moving membrane
    st = orc.get_state()
    a, dt = st.a, p.dtmd
    # the per-triangle normals of the streaming step (corners at t and t + dtmd)
    x = np.stack([a["x"], a["y"], a["z"]], 1)
    v = np.stack([a["vx"], a["vy"], a["vz"]], 1)
    t1, t2, t3 = T[:, 0], T[:, 1], T[:, 2]
    A1, B1, C1 = x[t1], x[t2], x[t3]
    A2, B2, C2 = A1 + v[t1] * dt, B1 + v[t2] * dt, C1 + v[t3] * dt
    X, Xdt = _cp(B1 - A1, C1 - A1), _cp(B2 - A2, C2 - A2)
    off, idx = st.llists()
    nx, ny, nz = int(Lx), int(Ly), int(Lz) + 1
    sx, sy, sz = a["sx"], a["sy"], a["sz"]
    fx, fy, fz = np.floor(sx).astype(int), np.floor(sy).astype(int), np.floor(sz + 1.0).astype(int)
    ok = (fx >= 0) & (fx < nx) & (fy >= 0) & (fy < ny) & (fz >= 0) & (fz < nz)
    pid = np.where(ok, (fx * ny + fy) * nz + fz, 0)
    listed = np.nonzero(ok & (off[pid + 1] > off[pid]))[0]
    band = (sx < 3.0) | (sx > Lx - 3.0) | (sy < 3.0) | (sy > Ly - 3.0)
    free, queued = [], 0
    for i in listed:
        ent = idx[off[pid[i]]:off[pid[i] + 1]]
        P = np.array([sx[i], sy[i], sz[i]])
        Q = np.array([sx[i] + a["svx"][i] * dt, sy[i] + a["svy"][i] * dt, sz[i] + a["svz"][i] * dt])
        d0, d1 = P - A1[ent], Q - A2[ent]
        bt = X[ent, 0] * d0[:, 0] + X[ent, 1] * d0[:, 1] + X[ent, 2] * d0[:, 2]
        bdt = Xdt[ent, 0] * d1[:, 0] + Xdt[ent, 1] * d1[:, 1] + Xdt[ent, 2] * d1[:, 2]
        flg = ((a["sindio"][i] == 1) & (bt < 0)) | ((a["sindio"][i] == 0) & (bt > 0))
        if band[i] or ((bt * bdt <= 0) & ~flg).any():
            queued += 1
        else:
            free.append(i)
    assert len(listed) > 10000 and free
    # the reference's loop on the oracle, particle by particle
    before = {k: a[k].copy() for k in ("sx", "sy", "sz", "svx", "svy", "svz")}
    L = orc.L
    for i in free:
        assert L.orc_reflection(orc.h, C.c_int64(int(i))) == 0.0
    after = orc.get_state().a
    for k in before:
        np.testing.assert_array_equal(after[k][free], before[k][free])
    # few particles need the full walk
    assert queued <= 0.05 * len(listed), (queued, len(listed))
