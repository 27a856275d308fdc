"""Generates the golden fixtures in this folder by running the REFERENCE's own code (petch's
threed.py / belen.py / chemistry.py, unmodified) on small seeded inputs, with the third-party
warp-lang replaced by warp_shim.py (a CPU stand-in: see its docstring for what it restates).

Point it at a checkout of the reference project (its root, the folder holding src/petch) with
--reference or the PETCH_REFERENCE environment variable:

    python tests/golden/make_golden.py --reference <path> [group ...]

groups: levelset surface flux radiosity options redep dda knudsen gmres electron

The fixtures are committed; tests read only the .npz files, never the reference.
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import warp_shim  # noqa: E402


def _reference_root(argv):
    """The reference checkout from --reference <path> (removed from argv) or PETCH_REFERENCE."""
    if "--reference" in argv:
        i = argv.index("--reference")
        if i + 1 >= len(argv):
            raise SystemExit("--reference needs a path")
        root = argv[i + 1]
        del argv[i:i + 2]
        return root
    root = os.environ.get("PETCH_REFERENCE")
    if not root:
        raise SystemExit("give the reference checkout with --reference <path> or PETCH_REFERENCE")
    return root


REF = _reference_root(sys.argv)
t3 = warp_shim.install(os.path.join(REF, "src", "petch"))


def _csg(nx, ny, nz, dx, Lx, Ly, sub_top, mask_th, width, hole):
    """make_trench_3d's analytic field and mask (threed.py:34-55), before skfmm."""
    xs, ys, zs = np.arange(nx) * dx, np.arange(ny) * dx, np.arange(nz) * dx
    X, Y, Z = np.meshgrid(xs, ys, zs, indexing="ij")
    mask_band = (Z >= sub_top) & (Z < sub_top + mask_th)
    if hole:
        opening = (X - Lx / 2) ** 2 + (Y - Ly / 2) ** 2 < (width / 2) ** 2
        r = np.sqrt((X - Lx / 2) ** 2 + (Y - Ly / 2) ** 2)
    else:
        opening = np.abs(X - Lx / 2) < width / 2
        r = np.abs(X - Lx / 2)
    d_sub = sub_top - Z
    d_slab = np.minimum(Z - sub_top, sub_top + mask_th - Z)
    d_mask = np.minimum(d_slab, r - width / 2.0)
    return np.maximum(d_sub, d_mask), mask_band & ~opening


def levelset():
    out = {}
    rng = np.random.default_rng(1234)
    cases = [
        # name, nx, ny, nz, dx, Lx, Ly, sub_top, mask_th, width, hole
        ("hole", 14, 14, 20, 0.25, 3.5, 3.5, 3.0, 0.75, 1.5, True),
        ("trench", 16, 6, 18, 0.15, 2.4, 0.9, 1.8, 0.3, 0.9, False),
    ]
    for name, nx, ny, nz, dx, Lx, Ly, sub_top, mask_th, width, hole in cases:
        phi_a, mask = _csg(nx, ny, nz, dx, Lx, Ly, sub_top, mask_th, width, hole)
        phi_a = phi_a.astype(np.float32)
        out[f"{name}_seed_args"] = np.array([nx, ny, nz, dx, Lx, Ly, sub_top, mask_th, width,
                                             float(hole)])
        out[f"{name}_csg"] = phi_a
        out[f"{name}_mask"] = mask
        band = 4 * dx + 2.0 * dx                         # run_etch_3d: reinit_fsm(phi, dx, band + 2dx)
        t0 = time.time()
        phi_r = t3.reinit_fsm(phi_a.astype(np.float64), dx, band)
        print(f"  reinit_fsm {name}: {time.time() - t0:.1f}s", flush=True)
        out[f"{name}_reinit_band"] = np.array([band])
        out[f"{name}_reinit"] = phi_r
        # advection on the redistanced field: F > 0 in the narrow band (as extend_velocity), a
        # sprinkle of exact zeros, mask cells re-pinned to the CSG field (mask_phi)
        phi1 = phi_r.astype(np.float32)
        F = np.where(np.abs(phi1) < 4 * dx, rng.uniform(0.0, 3.0, phi1.shape), 0.0)
        F[rng.random(phi1.shape) < 0.1] = 0.0
        F = F.astype(np.float32)
        dt, nsub = 0.02, 3
        t0 = time.time()
        adv = t3.advect_3d_gpu(phi1.astype(np.float64), F, mask, phi_a, dx, dt / nsub, nsub)
        print(f"  advect_3d_gpu {name}: {time.time() - t0:.1f}s", flush=True)
        out[f"{name}_F"] = F
        out[f"{name}_adv_args"] = np.array([dx, dt / nsub, nsub])
        out[f"{name}_advect"] = adv
        # the numpy twin (no mask) on the same input, one substep
        out[f"{name}_advect_np"] = t3.advect_3d(phi1.astype(np.float64), F.astype(np.float64),
                                                dx, dt / nsub)
    # a noisy field with exact zeros on nodes (sign(0) = +1, zero never an interface partner)
    nx, ny, nz, dx = 9, 8, 10, 0.2
    X, Y, Z = np.meshgrid(np.arange(nx) * dx, np.arange(ny) * dx, np.arange(nz) * dx, indexing="ij")
    phi = np.sqrt((X - 0.8) ** 2 + (Y - 0.7) ** 2 + (Z - 0.9) ** 2) - 0.55
    phi += rng.normal(0, 0.03, phi.shape)
    phi[rng.random(phi.shape) < 0.05] = 0.0
    phi = phi.astype(np.float32)
    out["noisy_phi"] = phi
    out["noisy_args"] = np.array([dx, 5 * dx, 3])
    out["noisy_reinit"] = t3.reinit_fsm(phi.astype(np.float64), dx, 5 * dx, n_iter=3)
    np.savez_compressed(os.path.join(HERE, "levelset.npz"), **out)


def _oracle():
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    import oracle.oracle as orc
    return orc


def _small_mesh(hole, nx=14, ny=14, nz=18, dx=0.25):
    """A small etched-feature mesh from the oracle's marching cubes (the reference's own MC is
    skimage/Warp, not restated): a masked hole or trench with a partly etched floor."""
    orc = _oracle()
    Lx, Ly, Lz = nx * dx, ny * dx, nz * dx
    sub_top, mask_th, width = 3.0, 0.75, 1.5
    phi_a, mask = orc.seed(nx, ny, nz, dx, Lx, Ly, sub_top, mask_th, width, hole)
    X, Y, Z = np.meshgrid(np.arange(nx) * dx, np.arange(ny) * dx, np.arange(nz) * dx, indexing="ij")
    r = np.sqrt((X - Lx / 2) ** 2 + (Y - Ly / 2) ** 2) if hole else np.abs(X - Lx / 2)
    # CSG difference: material minus a pit {r < width/2, z > 1.6} below the opening
    phi_a = np.minimum(phi_a, np.maximum(r - width / 2, 1.6 - Z))
    phi = orc.reinit(phi_a.astype(np.float32), dx, 6 * dx).astype(np.float32)
    geo = dict(Lx=Lx, Ly=Ly, Lz=Lz, dx=dx, sub_top=sub_top, mask_th=mask_th, trench_width=width,
               hole=hole, xs=np.arange(nx) * dx, ys=np.arange(ny) * dx, zs=np.arange(nz) * dx,
               phi=phi.astype(np.float64))
    m = orc.mesh_build(phi, dx, geo)
    return m, geo, phi


def surface():
    """Per-face arithmetic: adjacency, smoothing (host and device forms), Belen coverages,
    surface rates, faces_in_mask, yields, depth metrics."""
    import petch.belen as belen
    import petch.chemistry as chem
    out = {}
    rng = np.random.default_rng(7)
    m, geo, phi = _small_mesh(True)
    verts, faces = m.verts.astype(np.float32), m.faces
    out["mesh_verts"], out["mesh_faces"], out["mesh_normal"] = verts, faces, m.normal
    pairs = t3._edge_adjacency(faces)
    out["pairs"] = pairs
    fl = rng.uniform(0.0, 3.0, len(faces))
    out["smooth_in"] = fl
    for n_iter, alpha in ((1, 1.0), (2, 1.0), (1, 0.5)):
        out[f"smooth_host_{n_iter}_{alpha}"] = t3.smooth_flux(fl, m.normal, pairs, n_iter, alpha)
    prep = t3._smooth_prep_dev(verts, faces, pairs)
    out["prep_ww"] = np.asarray(prep["ww"])
    for alpha in (1.0, 0.5):
        out[f"smooth_dev_{alpha}"] = t3.smooth_flux_dev(t3.wp.array(fl, dtype=float), prep,
                                                        alpha=alpha).numpy()
    # chemistry on random per-face inputs
    F = 400
    m_i = rng.uniform(0.0, 1.5, F); m_F = rng.uniform(0.0, 2.0, F); m_O = rng.uniform(0.0, 2.0, F)
    cos_i = rng.uniform(-0.1, 1.1, F); cos_i[:5] = [0.0, 0.5, 1.0, 0.49999, -0.2]
    iy = tuple(rng.uniform(0.0, 5.0, F) for _ in range(3))
    is_mask = rng.random(F) < 0.2
    out.update(c_m_i=m_i, c_m_F=m_F, c_m_O=m_O, c_cos_i=cos_i, c_iy=np.stack(iy), c_is_mask=is_mask)
    par = dict(t3.PAR)
    for ya in ("cosine", "viennaps"):
        for ied in ("mean", "gauss", "bimodal"):
            p = dict(par, ied_mode=ied, rate_scale=0.7)
            fl_b = t3.DEFAULT_FLAGS.__class__(chemistry="belen", yield_angular=ya)
            fl_l = t3.DEFAULT_FLAGS.__class__(chemistry="langmuir", yield_angular=ya)
            out[f"yields_{ied}"] = np.array(chem._yields(p))
            thF, thO = t3._belen_coverages(m_i, m_F, m_O, cos_i, p, fl_b)
            out[f"cov_{ya}_{ied}"] = np.stack([thF, thO])
            out[f"rate_belen_{ya}_{ied}"] = belen.surface_rate_belen(m_i, m_F, m_O, cos_i, is_mask,
                                                                     p, fl_b)
            out[f"rate_langmuir_{ya}_{ied}"] = chem.surface_rate_langmuir(m_i, m_F, m_O, cos_i,
                                                                          is_mask, p, fl_l)
            p2 = dict(p, _ion_yield=iy)
            thF, thO = t3._belen_coverages(m_i, m_F, m_O, cos_i, p2, fl_b)
            out[f"covy_{ya}_{ied}"] = np.stack([thF, thO])
            out[f"ratey_belen_{ya}_{ied}"] = belen.surface_rate_belen(m_i, m_F, m_O, cos_i,
                                                                      is_mask, p2, fl_b)
    # faces_in_mask: random centroids plus exact band edges
    for hole in (True, False):
        g = dict(Lx=4.0, Ly=3.0, sub_top=2.0)
        c = np.stack([rng.uniform(0, 4, 300), rng.uniform(0, 3, 300), rng.uniform(1.5, 3.0, 300)], 1)
        c[:4, 2] = [2.0, 2.5, 2.5 - 1e-12, 1.9999999]
        c[4:8, 0] = [2.0 - 0.6, 2.0 + 0.6, 2.0, 2.6]
        key = "hole" if hole else "trench"
        out[f"fim_{key}_c"] = c
        out[f"fim_{key}"] = t3.faces_in_mask(c, g, 0.5, 1.2, hole=hole)
    # depth metrics on etched level sets
    for hole in (True, False):
        mm, g, ph = _small_mesh(hole)
        key = "hole" if hole else "trench"
        g = dict(g, phi=ph.astype(np.float64))
        out[f"depth_{key}_phi"] = ph
        out[f"depth_{key}"] = np.array([t3.center_depth_3d(g), t3.max_depth_3d(g),
                                        t3.center_depth_3d(g, half=0.4)])
    np.savez_compressed(os.path.join(HERE, "surface.npz"), **out)


def _mean_se(fn, seeds):
    runs = np.stack([fn(s) for s in seeds])
    return runs.mean(0), runs.std(0, ddof=1) / np.sqrt(len(seeds))


def flux():
    """Monte-Carlo kernels of the reference (shim-executed) on small meshes: per-face means and
    standard errors over independent seeds.  Sources come from the reference's host path
    (_source3d with sampling='pseudo', threed.py:410-438), whose random stream is independent of
    the trace kernel's.  (On its CUDA path the reference seeds _gen_source and the trace kernel
    with the same (seed, thread) stream, so a ray's first sticking / re-emission draws repeat its
    source draws; that correlation is not reproduced.)"""
    out = {}
    wp = t3.wp
    rng = np.random.default_rng(11)
    for hole in (True, False):
        key = "hole" if hole else "trench"
        m, geo, phi = _small_mesh(hole, nx=10, ny=10, nz=14, dx=0.3)
        verts, faces = m.verts, m.faces
        F = len(faces)
        mesh = wp.Mesh(points=wp.array(verts, dtype=wp.vec3),
                       indices=wp.array(faces.flatten(), dtype=wp.int32))
        Lx, Ly, Lz = geo['Lx'], geo['Ly'], geo['Lz']
        periodic = 0 if hole else 1
        z_src = Lz - geo['dx']
        out[f"{key}_verts"], out[f"{key}_faces"] = verts, faces
        out[f"{key}_geo"] = np.array([Lx, Ly, Lz, geo['dx'], periodic])
        bare = rng.uniform(0.2, 1.0, F)
        out[f"{key}_bare"] = bare
        n = 6000
        par = dict(t3.PAR)

        def src(kind, sd, sigma):
            o, d = t3._source3d(kind, n, Lx, Ly, z_src, sigma, 'pseudo',
                                np.random.default_rng(sd), sd)
            return wp.array(o, dtype=wp.vec3), wp.array(d, dtype=wp.vec3)

        def neutral(sd):
            o, d = src('neutral', sd, 0.0)
            f = wp.zeros(F, dtype=float)
            wp.launch(t3._trace3d_cov_rr, dim=n, inputs=[mesh.id, o, d, wp.array(bare), 0.7, sd, f,
                                                         Lx, Ly, Lz, periodic])
            return f.numpy() / n

        def ion(sd):
            o, d = src('ion', sd, par['ion_ang_sigma'])
            arrs = [wp.zeros(F, dtype=float) for _ in range(5)]
            inflect, minang, n_l = par['inflectAngle'], par['minAngle'], par['n_l']
            A_en = 1.0 / (1.0 + n_l * (1.5707963 / inflect - 1.0))
            wp.launch(t3._trace3d_ion_yield, dim=n, inputs=[
                mesh.id, o, d, sd, par['Emean'], par['Esig'], par['A_sp'], par['Eth_sp'], par['B_sp'],
                par['A_ie'], par['Eth_ie'], par['A_p'], par['Eth_p'], inflect, minang, n_l, A_en,
                min(par['Eth_ie'], par['Eth_sp']), par['thetaRMin'], par['thetaRMax'],
                Lx, Ly, Lz, periodic, *arrs])
            return np.stack([a.numpy() for a in arrs]) / n

        def legacy(sd):
            o, d = src('neutral', sd, 0.0)
            f, a = wp.zeros(F, dtype=float), wp.zeros(F, dtype=float)
            wp.launch(t3._trace3d, dim=n, inputs=[mesh.id, o, d, 0.2, 12, sd, 0, 0.34, 0.8, f, a])
            return np.stack([f.numpy(), a.numpy()]) / n

        for name, fn in (("neutral", neutral), ("ion", ion), ("legacy", legacy)):
            t0 = time.time()
            mean, se = _mean_se(fn, range(100, 108))
            print(f"  {key} {name}: {time.time() - t0:.1f}s", flush=True)
            out[f"{key}_{name}_mean"], out[f"{key}_{name}_se"] = mean, se
            out[f"{key}_{name}_n"] = np.array([n * 8])
    np.savez_compressed(os.path.join(HERE, "flux.npz"), **out)


def radiosity():
    """mc_flux_3d_radiosity (threed.py:923-991) run unmodified on small meshes.  For one seed per
    case the form-factor hits of its _trace_ff launch are recorded with the ion results, so the
    deterministic part (matrix assembly, Jacobi solves, coverage fixed point) can be replayed
    exactly; over 8 seeds the per-face means and standard errors of (m_i, m_F, m_O) pin the
    estimator statistically.  _gas_normals is recorded on the same meshes."""
    out = {}
    wp = t3.wp
    real_launch = wp.launch
    rec = {}

    def launch(k, dim, device=None, inputs=()):
        real_launch(k, dim, device=device, inputs=inputs)
        if k is t3._trace_ff:
            rec['hit'] = np.asarray(inputs[3]).astype(np.int32).copy()

    wp.launch = launch
    try:
        cases = (("hole", True, True), ("trench", False, True), ("hole_legacy", True, False))
        for key, hole, faithful in cases:
            m, geo, phi = _small_mesh(hole, nx=10, ny=10, nz=14, dx=0.3)
            verts = m.verts.astype(np.float32)
            faces = m.faces
            v64 = verts.astype(np.float64)[faces]
            centroids = v64.mean(axis=1)
            areas = 0.5 * np.linalg.norm(np.cross(v64[:, 1] - v64[:, 0], v64[:, 2] - v64[:, 0]),
                                         axis=1)
            geo = dict(geo, phi=phi.astype(np.float64))
            mesh = wp.Mesh(points=wp.array(verts, dtype=wp.vec3),
                           indices=wp.array(faces.flatten(), dtype=wp.int32))
            par = dict(t3.PAR, periodic_y=0 if hole else 1)
            flags = t3.DEFAULT_FLAGS.__class__(
                chemistry="belen" if faithful else "langmuir", yield_angular="viennaps",
                ion_reflection=faithful, coverage_sticking=True, neutral_transport="radiosity")
            out[f"{key}_verts"], out[f"{key}_faces"] = verts, faces
            out[f"{key}_phi"] = phi.astype(np.float32)
            out[f"{key}_geo"] = np.array([geo['Lx'], geo['Ly'], geo['Lz'], geo['dx'],
                                          par['periodic_y']])
            out[f"{key}_gas_normals"] = t3._gas_normals(verts, faces, centroids, geo)
            n_ion = 3000

            def run(sd):
                p = dict(par)
                t0 = time.time()
                r = t3.mc_flux_3d_radiosity(mesh, verts, faces, centroids, areas, geo, p,
                                            n_ion=n_ion, n_ff=64, seed=sd, flags=flags)
                print(f"  {key} seed {sd}: {time.time() - t0:.1f}s", flush=True)
                return r, p

            (m_i, m_F, m_O, cos_i), p = run(100)
            out[f"{key}_hit"] = rec['hit']
            out[f"{key}_m_i"], out[f"{key}_cos_i"] = m_i, cos_i
            out[f"{key}_m_F"], out[f"{key}_m_O"] = m_F, m_O
            if faithful:
                out[f"{key}_ion_yield"] = np.stack(p['_ion_yield'])
            if key == "hole_legacy":
                continue

            def stats(sd):
                (mi, mF, mO, _), _ = run(sd)
                return np.stack([mi, mF, mO])

            mean, se = _mean_se(stats, range(200, 208))
            out[f"{key}_mean"], out[f"{key}_se"] = mean, se
    finally:
        wp.launch = real_launch
    np.savez_compressed(os.path.join(HERE, "radiosity.npz"), **out)


def options():
    """run_etch_3d's non-default level-set options on the reference's own functions: the PDE
    reinit (reinit_gpu, reinit_method='gpu') and the nearest-centroid extension
    (extend_velocity_3d, extend != 'gpu')."""
    out = {}
    rng = np.random.default_rng(99)
    for name, nx, ny, nz, dx, Lx, Ly, sub_top, mask_th, width, hole in (
            ("hole", 12, 12, 16, 0.25, 3.0, 3.0, 2.5, 0.75, 1.5, True),
            ("trench", 14, 6, 16, 0.15, 2.1, 0.9, 1.5, 0.3, 0.9, False)):
        phi_a, _ = _csg(nx, ny, nz, dx, Lx, Ly, sub_top, mask_th, width, hole)
        phi_a = (phi_a + rng.normal(0.0, 0.02 * dx, phi_a.shape)).astype(np.float32)
        out[f"{name}_pde_in"] = phi_a
        out[f"{name}_pde_dx"] = np.array([dx])
        t0 = time.time()
        out[f"{name}_pde_out"] = t3.reinit_gpu(phi_a.astype(np.float64), dx)
        print(f"  reinit_gpu {name}: {time.time() - t0:.1f}s", flush=True)
    m, geo, phi = _small_mesh(True)
    v64 = m.verts.astype(np.float32).astype(np.float64)[m.faces]
    centroids = v64.mean(axis=1)
    V = rng.uniform(0.0, 2.0, len(m.faces))
    band = 4 * geo['dx']
    g = dict(geo, phi=phi.astype(np.float64))
    out["ext_phi"], out["ext_centroids"], out["ext_V"] = phi, centroids, V
    out["ext_verts"], out["ext_faces"] = m.verts.astype(np.float32), m.faces
    out["ext_args"] = np.array([geo['dx'], band])
    out["ext_Fs"] = t3.extend_velocity_3d(V, centroids, g, band)
    np.savez_compressed(os.path.join(HERE, "options.npz"), **out)


def redep():
    """mc_redep_3d (threed.py:1582-1605) run unmodified on small meshes: per-face means and
    standard errors of the redeposited flux density over 8 seeds, for a random source rate with
    some non-etching faces."""
    out = {}
    wp = t3.wp
    rng = np.random.default_rng(21)
    for key, hole in (("hole", True), ("trench", False)):
        m, geo, phi = _small_mesh(hole, nx=10, ny=10, nz=14, dx=0.3)
        verts = m.verts.astype(np.float32)
        faces = m.faces
        v64 = verts.astype(np.float64)[faces]
        centroids = v64.mean(axis=1)
        areas = 0.5 * np.linalg.norm(np.cross(v64[:, 1] - v64[:, 0], v64[:, 2] - v64[:, 0]),
                                     axis=1)
        geo = dict(geo, phi=phi.astype(np.float64))
        fn = t3._gas_normals(verts, faces, centroids, geo)
        mesh = wp.Mesh(points=wp.array(verts, dtype=wp.vec3),
                       indices=wp.array(faces.flatten(), dtype=wp.int32))
        V = rng.uniform(0.0, 2.0, len(faces))
        V[rng.random(len(faces)) < 0.3] = 0.0
        out[f"{key}_verts"], out[f"{key}_faces"], out[f"{key}_phi"] = verts, faces, phi
        out[f"{key}_V"], out[f"{key}_gas_normals"] = V, fn
        out[f"{key}_geo"] = np.array([geo['Lx'], geo['Ly'], geo['Lz'], geo['dx']])
        n = 4000

        def run(sd):
            t0 = time.time()
            r = t3.mc_redep_3d(mesh, centroids, areas, fn, V, n_redep=n, s_redep=0.5, seed=sd)
            print(f"  {key} seed {sd}: {time.time() - t0:.1f}s", flush=True)
            return r

        mean, se = _mean_se(run, range(100, 108))
        out[f"{key}_mean"], out[f"{key}_se"] = mean, se
        out[f"{key}_n"] = np.array([n])
    np.savez_compressed(os.path.join(HERE, "redep.npz"), **out)


def dda():
    """The DDA neutral transport (petch/dda.py, wired as mc_flux_3d_dda, threed.py:1211-1244) run
    unmodified on small meshes: single launches of _dda_gather_kernel (the direct view with a zero
    re-emission field, and one pass over a random re-emission field), dda_neutral_flux for a random
    sticking field at several direction / iteration counts, and mc_flux_3d_dda itself with its
    ion results recorded so the deterministic part can be replayed."""
    import petch.dda as dda_mod
    out = {}
    wp = t3.wp
    rng = np.random.default_rng(77)
    for key, hole in (("hole", True), ("trench", False)):
        m, geo, phi = _small_mesh(hole, nx=10, ny=10, nz=14, dx=0.3)
        nx, ny, nz = phi.shape
        dx = geo['dx']
        periodic = 0 if hole else 1
        verts = m.verts.astype(np.float32)
        faces = m.faces
        v64 = verts.astype(np.float64)[faces]
        centroids = v64.mean(axis=1)
        areas = 0.5 * np.linalg.norm(np.cross(v64[:, 1] - v64[:, 0], v64[:, 2] - v64[:, 0]),
                                     axis=1)
        geo = dict(geo, phi=phi.astype(np.float64))
        fn = t3._gas_normals(verts, faces, centroids, geo)
        F = len(faces)
        out[f"{key}_verts"], out[f"{key}_faces"], out[f"{key}_phi"] = verts, faces, phi
        out[f"{key}_centroids"], out[f"{key}_areas"], out[f"{key}_gas_normals"] = (
            centroids, areas, fn)
        out[f"{key}_geo"] = np.array([geo['Lx'], geo['Ly'], geo['Lz'], dx, periodic])
        zs = geo['zs']
        z_top = zs[-1] - 0.5 * dx
        max_steps = (int((z_top - zs[0]) / dx) + 4) * (3 if periodic else 1)

        # single launches of the gather kernel with the 128-direction sphere (dda_n_dir = 64)
        dirs, w = dda_mod.fib_sphere(128)
        out[f"{key}_dirs"] = dirs
        remit = np.zeros(nx * ny * nz)
        solid = (phi > 0).ravel()
        remit[solid] = rng.uniform(0.0, 1.0, int(solid.sum()))
        out[f"{key}_remit"] = remit

        def gather(rem, src):
            o = wp.zeros(F, dtype=wp.float32)
            wp.launch(dda_mod._dda_gather_kernel, dim=F,
                      inputs=[wp.array(np.ascontiguousarray(phi, dtype=np.float32)),
                              wp.array(centroids.astype(np.float32), dtype=wp.vec3),
                              wp.array(fn.astype(np.float32), dtype=wp.vec3),
                              wp.array(dirs.astype(np.float32), dtype=wp.vec3),
                              wp.array(w.astype(np.float32)),
                              wp.array(rem.astype(np.float32)), float(dx), float(z_top),
                              float(src), int(max_steps), nx, ny, nz, periodic, o])
            return o.numpy().astype(np.float64)

        t0 = time.time()
        out[f"{key}_direct"] = gather(np.zeros(nx * ny * nz), 1.0)
        out[f"{key}_remit_pass"] = gather(remit, 0.0)
        print(f"  {key} gathers: {time.time() - t0:.1f}s", flush=True)

        # dda_neutral_flux for a random sticking field
        s_face = rng.uniform(0.05, 1.0, F)
        out[f"{key}_s_face"] = s_face
        for n_dir, n_re in ((16, 12), (8, 1), (8, 2), (8, 5)):
            t0 = time.time()
            out[f"{key}_flux_{n_dir}_{n_re}"] = dda_mod.dda_neutral_flux(
                phi, dx, zs, centroids, fn, s_face, n_dir=n_dir, n_reemit=n_re,
                face_areas=np.maximum(areas, 1e-9), periodic_y=periodic)
            print(f"  {key} dda_neutral_flux({n_dir}, {n_re}): {time.time() - t0:.1f}s",
                  flush=True)

        # mc_flux_3d_dda: faithful ions, 16 directions, 12 re-emission passes, 4 coverage rounds
        mesh = wp.Mesh(points=wp.array(verts, dtype=wp.vec3),
                       indices=wp.array(faces.flatten(), dtype=wp.int32))
        par = dict(t3.PAR, periodic_y=periodic, dda_n_dir=8, dda_n_reemit=12)
        flags = t3.DEFAULT_FLAGS.__class__(chemistry="belen", yield_angular="viennaps",
                                           ion_reflection=True, coverage_sticking=True,
                                           neutral_transport="dda")
        p = dict(par)
        t0 = time.time()
        m_i, m_F, m_O, cos_i = t3.mc_flux_3d_dda(mesh, verts, faces, centroids, areas, geo, p,
                                                 n_ion=3000, seed=100, flags=flags)
        print(f"  {key} mc_flux_3d_dda: {time.time() - t0:.1f}s", flush=True)
        out[f"{key}_m_i"], out[f"{key}_cos_i"] = m_i, cos_i
        out[f"{key}_m_F"], out[f"{key}_m_O"] = m_F, m_O
        out[f"{key}_ion_yield"] = np.stack(p['_ion_yield'])
    np.savez_compressed(os.path.join(HERE, "dda.npz"), **out)


def knudsen():
    """The Knudsen conductance tail (petch/knudsen.py, wired as mc_flux_3d_knudsen,
    threed.py:1149-1208) and the charging hooks (_apply_hg_charging :1046-1110,
    _apply_floor_charge_throttle :1112-1147) run unmodified on small meshes: slice geometry,
    conductance profiles for random sinks (scalar and per-slice loss scales), knudsen_face_flux
    with and without the footprint filter and the front loss, mc_flux_3d_knudsen with recorded
    ions (local and field sinks, with and without surface_charging), and both hooks on recorded
    inputs."""
    import petch.knudsen as kn
    out = {}
    wp = t3.wp
    rng = np.random.default_rng(31)
    for key, hole, deep in (("hole", True, False), ("trench", False, False),
                            ("hole_deep", True, True), ("trench_deep", False, True)):
        nz = 22 if deep else 14
        m, geo, phi = _small_mesh(hole, nx=10, ny=10, nz=nz, dx=0.3)
        if deep:                       # a deeper pit: material minus {r < w/2, z > 0.45}
            orc = _oracle()
            nx, ny = 10, 10
            dx, Lx, Ly = 0.3, 3.0, 3.0
            sub_top = 5.4
            phi_a, _ = orc.seed(nx, ny, nz, dx, Lx, Ly, sub_top, 0.75, 1.5, hole)
            X, Y, Z = np.meshgrid(np.arange(nx) * dx, np.arange(ny) * dx, np.arange(nz) * dx,
                                  indexing="ij")
            r = np.sqrt((X - Lx / 2) ** 2 + (Y - Ly / 2) ** 2) if hole else np.abs(X - Lx / 2)
            phi_a = np.minimum(phi_a, np.maximum(r - 0.75, 0.45 - Z))
            phi = orc.reinit(phi_a.astype(np.float32), dx, 6 * dx).astype(np.float32)
            geo = dict(geo, sub_top=sub_top, Lz=nz * dx, zs=np.arange(nz) * dx,
                       phi=phi.astype(np.float64))
            m = orc.mesh_build(phi, dx, geo)
        dx, sub_top = geo['dx'], geo['sub_top']
        periodic = 0 if hole else 1
        shape = "via" if hole else "trench"
        verts = m.verts.astype(np.float32)
        faces = m.faces
        v64 = verts.astype(np.float64)[faces]
        centroids = v64.mean(axis=1)
        areas = 0.5 * np.linalg.norm(np.cross(v64[:, 1] - v64[:, 0], v64[:, 2] - v64[:, 0]),
                                     axis=1)
        geo = dict(geo, phi=phi.astype(np.float64))
        fn = t3._gas_normals(verts, faces, centroids, geo)
        F = len(faces)
        zs = geo['zs']
        A = np.maximum(areas, 1e-9)
        out[f"{key}_verts"], out[f"{key}_faces"], out[f"{key}_phi"] = verts, faces, phi
        out[f"{key}_centroids"], out[f"{key}_areas"], out[f"{key}_gas_normals"] = (
            centroids, areas, fn)
        out[f"{key}_geo"] = np.array([geo['Lx'], geo['Ly'], geo['Lz'], dx, periodic, sub_top,
                                      geo['trench_width']])
        area, perim = kn.slice_geometry(phi.astype(np.float64), zs, dx, sub_top, shape)
        out[f"{key}_slice_area"], out[f"{key}_slice_perim"] = area, perim
        loss = rng.uniform(0.0, 0.3, nz) * (rng.random(nz) < 0.7)
        out[f"{key}_loss"] = loss
        out[f"{key}_profile_scalar"] = kn.conductance_profile(phi.astype(np.float64), zs, dx,
                                                              sub_top, shape, loss, 1.85)
        ls = rng.uniform(0.5, 3.0, nz)
        out[f"{key}_ls"] = ls
        out[f"{key}_profile_array"] = kn.conductance_profile(phi.astype(np.float64), zs, dx,
                                                             sub_top, shape, loss, ls)
        s_face = rng.uniform(0.0, 1.0, F)
        out[f"{key}_s_face"] = s_face
        ctr = (0.5 * geo['Lx'], 0.5 * geo['Ly'])
        hw = 0.5 * geo['trench_width']
        kw = dict(center=ctr, half_width=hw)
        out[f"{key}_kff_plain"] = kn.knudsen_face_flux(phi.astype(np.float64), zs, dx, sub_top,
                                                       shape, centroids, fn[:, 2], A, geo['Ly'],
                                                       s_face, 2.9)
        out[f"{key}_kff_foot"] = kn.knudsen_face_flux(phi.astype(np.float64), zs, dx, sub_top,
                                                      shape, centroids, fn[:, 2], A, geo['Ly'],
                                                      s_face, 2.9, **kw)
        out[f"{key}_kff_front"] = kn.knudsen_face_flux(phi.astype(np.float64), zs, dx, sub_top,
                                                       shape, centroids, fn[:, 2], A, geo['Ly'],
                                                       s_face, 2.0, front_loss=True, band_W=1.0,
                                                       pass_frac=0.3, ar_pass=0.7, **kw)

        mesh = wp.Mesh(points=wp.array(verts, dtype=wp.vec3),
                       indices=wp.array(faces.flatten(), dtype=wp.int32))
        runs = (("local", dict(), dict()), ("field", dict(knudsen_sink='field'), dict()),
                ("front", dict(knudsen_front_band_W=1.0, knudsen_passive_frac=0.3,
                               knudsen_front_ar_pass=0.7), dict(knudsen_front_loss=True)),
                ("hg", dict(), dict(surface_charging="hg")),
                ("petch", dict(), dict(surface_charging="petch")))
        for name, pkw, fkw in runs:
            par = dict(t3.PAR, periodic_y=periodic, **pkw)
            flags = t3.DEFAULT_FLAGS.__class__(chemistry="belen", yield_angular="viennaps",
                                               ion_reflection=True, coverage_sticking=True,
                                               neutral_transport="knudsen", **fkw)
            p = dict(par)
            t0 = time.time()
            m_i, m_F, m_O, cos_i = t3.mc_flux_3d_knudsen(mesh, verts, faces, centroids, areas,
                                                         geo, p, n_ion=3000, seed=100,
                                                         flags=flags)
            print(f"  {key} mc_flux_3d_knudsen[{name}]: {time.time() - t0:.1f}s", flush=True)
            out[f"{key}_{name}_m_i"], out[f"{key}_{name}_cos_i"] = m_i, cos_i
            out[f"{key}_{name}_m_F"], out[f"{key}_{name}_m_O"] = m_F, m_O
            out[f"{key}_{name}_ion_yield"] = np.stack(p['_ion_yield'])

        # the hooks on recorded inputs
        m_i = rng.uniform(0.0, 1.5, F)
        iy = tuple(rng.uniform(0.0, 3.0, F) for _ in range(3))
        out[f"{key}_hook_m_i"], out[f"{key}_hook_iy"] = m_i, np.stack(iy)
        for mode in ("hg", "petch"):
            par = dict(t3.PAR, _ion_yield=iy)
            flags = t3.DEFAULT_FLAGS.__class__(chemistry="belen", surface_charging=mode)
            mi2 = t3._apply_hg_charging(m_i, par, flags, centroids, fn[:, 2], A, geo)
            out[f"{key}_{mode}_hook_m_i"] = mi2
            out[f"{key}_{mode}_hook_iy"] = np.stack(par['_ion_yield'])
        par = dict(t3.PAR, _ion_yield=iy)
        mi2 = t3._apply_floor_charge_throttle(m_i, par, verts, faces, geo)
        out[f"{key}_throttle_m_i"] = mi2
        out[f"{key}_throttle_iy"] = np.stack(par['_ion_yield'])
    np.savez_compressed(os.path.join(HERE, "knudsen.npz"), **out)


def gmres():
    """mc_flux_3d_radiosity with radiosity_solver='gmres' (threed.py:964-985: scipy's gmres on
    (I - M) G = D, rtol 1e-3, restart 12, maxiter 40, Jacobi on failure) on the radiosity group's
    meshes at its recorded seed: the form-factor hits and ion results are recorded with the
    solution, so the solve can be replayed."""
    out = {}
    wp = t3.wp
    real_launch = wp.launch
    rec = {}

    def launch(k, dim, device=None, inputs=()):
        real_launch(k, dim, device=device, inputs=inputs)
        if k is t3._trace_ff:
            rec['hit'] = np.asarray(inputs[3]).astype(np.int32).copy()

    wp.launch = launch
    try:
        for key, hole in (("hole", True), ("trench", False)):
            m, geo, phi = _small_mesh(hole, nx=10, ny=10, nz=14, dx=0.3)
            verts = m.verts.astype(np.float32)
            faces = m.faces
            v64 = verts.astype(np.float64)[faces]
            centroids = v64.mean(axis=1)
            areas = 0.5 * np.linalg.norm(np.cross(v64[:, 1] - v64[:, 0], v64[:, 2] - v64[:, 0]),
                                         axis=1)
            geo = dict(geo, phi=phi.astype(np.float64))
            mesh = wp.Mesh(points=wp.array(verts, dtype=wp.vec3),
                           indices=wp.array(faces.flatten(), dtype=wp.int32))
            for bE, tag in ((0.7, "a"), (0.05, "b")):    # b: high albedo, where Jacobi lags
                par = dict(t3.PAR, periodic_y=0 if hole else 1, radiosity_solver="gmres",
                           betaE=bE)
                flags = t3.DEFAULT_FLAGS.__class__(chemistry="belen", yield_angular="viennaps",
                                                   ion_reflection=True, coverage_sticking=True,
                                                   neutral_transport="radiosity")
                p = dict(par)
                t0 = time.time()
                m_i, m_F, m_O, cos_i = t3.mc_flux_3d_radiosity(mesh, verts, faces, centroids,
                                                               areas, geo, p, n_ion=3000, n_ff=64,
                                                               seed=100, flags=flags)
                print(f"  {key}/{tag} gmres: {time.time() - t0:.1f}s", flush=True)
                out[f"{key}_{tag}_hit"] = rec['hit']
                out[f"{key}_{tag}_m_i"], out[f"{key}_{tag}_cos_i"] = m_i, cos_i
                out[f"{key}_{tag}_m_F"], out[f"{key}_{tag}_m_O"] = m_F, m_O
                out[f"{key}_{tag}_ion_yield"] = np.stack(p['_ion_yield'])
                out[f"{key}_{tag}_betaE"] = np.array([bE])
            out[f"{key}_verts"], out[f"{key}_faces"] = verts, faces
            out[f"{key}_phi"] = phi.astype(np.float32)
    finally:
        wp.launch = real_launch
    np.savez_compressed(os.path.join(HERE, "gmres.npz"), **out)


def electron():
    """The electron-shadowing charge model of mc_flux_3d_coupled (threed.py:847-868) run
    unmodified: (1) its electron trace (_source3d('ion', ..., e_ang_sigma) + _trace3d_cov_rr with
    bare = 1, beta = 1) over 8 seeds, per-face mean and standard error; (2) mc_flux_3d_coupled with
    surface_charging and charge_alpha > 0 (faithful and legacy ions), with every trace launch's
    tallies recorded, so the normalisation, the charging factor and the coverage fixed point can
    be replayed exactly from them."""
    out = {}
    wp = t3.wp
    real_launch = wp.launch
    rec = []

    def launch(k, dim, device=None, inputs=()):
        real_launch(k, dim, device=device, inputs=inputs)
        if k is t3._trace3d_cov_rr:
            rec.append(("rr", int(inputs[5]), float(inputs[4]), np.asarray(inputs[6]).copy()))
        elif k is t3._trace3d_ion_yield:
            rec.append(("ion", int(inputs[3]), 0.0,
                        np.stack([np.asarray(a).copy() for a in inputs[-5:]])))
        elif k is t3._trace3d:
            rec.append(("legacy", int(inputs[5]), 0.0,
                        np.stack([np.asarray(a).copy() for a in inputs[-2:]])))

    for hole in (True, False):
        key = "hole" if hole else "trench"
        m, geo, phi = _small_mesh(hole, nx=10, ny=10, nz=14, dx=0.3)
        verts = m.verts.astype(np.float32)
        faces = m.faces
        F = len(faces)
        v64 = verts.astype(np.float64)[faces]
        areas = 0.5 * np.linalg.norm(np.cross(v64[:, 1] - v64[:, 0], v64[:, 2] - v64[:, 0]),
                                     axis=1)
        mesh = wp.Mesh(points=wp.array(verts, dtype=wp.vec3),
                       indices=wp.array(faces.flatten(), dtype=wp.int32))
        Lx, Ly, Lz = geo['Lx'], geo['Ly'], geo['Lz']
        periodic = 0 if hole else 1
        out[f"{key}_verts"], out[f"{key}_faces"], out[f"{key}_areas"] = verts, faces, areas
        out[f"{key}_geo"] = np.array([Lx, Ly, Lz, geo['dx'], periodic])
        n = 6000

        def etrace(sd):
            o, d = t3._source3d('ion', n, Lx, Ly, Lz - geo['dx'], 0.5, 'pseudo',
                                np.random.default_rng(sd), sd)
            f = wp.zeros(F, dtype=float)
            wp.launch(t3._trace3d_cov_rr, dim=n, inputs=[
                mesh.id, wp.array(o, dtype=wp.vec3), wp.array(d, dtype=wp.vec3),
                wp.array(np.ones(F, np.float32), dtype=float), 1.0, sd, f, Lx, Ly, Lz, periodic])
            return f.numpy() / n

        t0 = time.time()
        mean, se = _mean_se(etrace, range(100, 108))
        print(f"  {key} electrons: {time.time() - t0:.1f}s", flush=True)
        out[f"{key}_electron_mean"], out[f"{key}_electron_se"] = mean, se
        out[f"{key}_electron_n"] = np.array([n * 8])

        wp.launch = launch
        try:
            for tag, faithful in (("faithful", True), ("legacy", False)):
                par = dict(t3.PAR, periodic_y=periodic, charge_alpha=0.6, eFlux=1.3)
                flags = t3.DEFAULT_FLAGS.__class__(
                    chemistry="belen", yield_angular="viennaps", ion_reflection=faithful,
                    coverage_sticking=True, surface_charging=True)
                rec.clear()
                p = dict(par)
                t0 = time.time()
                m_i, m_F, m_O, cos_i, bare = t3.mc_flux_3d_coupled(
                    mesh, verts, faces, areas, geo, p, n_ion=3000, n_neu=3000, seed=100,
                    flags=flags)
                print(f"  {key} mc_flux_3d_coupled[{tag}]: {time.time() - t0:.1f}s", flush=True)
                kinds = [r[0] for r in rec]
                seeds = [r[1] for r in rec]
                assert kinds[0] == ("ion" if faithful else "legacy") and seeds[1] == 100 * 9 + 7
                out[f"{key}_{tag}_ion_raw"] = rec[0][3]
                out[f"{key}_{tag}_electron_raw"] = rec[1][3]
                out[f"{key}_{tag}_neutral_raw"] = np.stack([r[3] for r in rec[2:]])
                out[f"{key}_{tag}_neutral_seed"] = np.array(seeds[2:])
                out[f"{key}_{tag}_neutral_beta"] = np.array([r[2] for r in rec[2:]])
                out[f"{key}_{tag}_m_i"], out[f"{key}_{tag}_m_F"] = m_i, m_F
                out[f"{key}_{tag}_m_O"], out[f"{key}_{tag}_cos_i"] = m_O, cos_i
                out[f"{key}_{tag}_bare"] = bare
                if faithful:
                    out[f"{key}_{tag}_ion_yield"] = np.stack(p['_ion_yield'])
        finally:
            wp.launch = real_launch
    np.savez_compressed(os.path.join(HERE, "electron.npz"), **out)


GROUPS = {"levelset": levelset, "surface": surface, "flux": flux, "radiosity": radiosity,
          "options": options, "redep": redep, "dda": dda, "knudsen": knudsen, "gmres": gmres,
          "electron": electron}

if __name__ == "__main__":
    for g in (sys.argv[1:] or list(GROUPS)):
        print(g, flush=True)
        GROUPS[g]()
