"""Generate the golden fixtures in tests/golden/ from DFTBaby's own code.

DFTBaby is Python 2 code, so its pure-numpy modules on the LR-TD-DFTB path are
loaded through a mechanical py2->py3 shim (print statements become calls,
``iteritems``/``xrange``/``has_key`` are renamed; nothing else changes) into a
throw-away package under a temporary directory.  Modules run this way:

* ``DFTB/Solver.py``            Casida, HermitianDavidson, nonHermitianDavidson, _ApBv, _AmBv
* ``DFTB/GammaApproximation.py`` gaussian_decay, GammaGaussian, GammaGaussianLC, GammaMatrix
* ``DFTB/ConvAcceleration.py``   DIIS_80
* ``DFTB/ExcGradients.py``       Gradients.gradient (gradient_lc / gradient_nolc) with its
                                 Python F and F^lr operators (SLAKO_IMPLEMENTATION = "PY");
                                 gradS/gradH0 and the repulsive potentials are supplied by
                                 the oracle, the gamma gradients come from DFTBaby's own
                                 GammaMatrix.gamma_AOwise

The Slater-Koster angular rules (``DFTB/extensions/slako_transformations_lmax2.f90``,
``..._dipole_lmax2.f90`` and ``..._grad_lmax2.f90``) are Fortran ``SELECT CASE`` tables whose
right-hand sides are also valid Python expressions; they are evaluated here for
random directions and table values.

Inputs of the solver fixtures (transition charges, gamma matrices, orbital
energy differences) come from a small seeded polyene; they are stored in the
fixtures next to the reference outputs, so the tests feed identical inputs to
the code under test.

Coupling and surface-hopping fixtures (``couplings.npz``) run single method texts of
``DFTB/ScalarCoupling.py`` (ci_overlap, with the AO overlap supplied), ``DFTB/PES.py``
(getScalarCouplings, with the CI overlaps supplied) and ``DFTB/Dynamics/SurfaceHopping.py``
(local diabatization, hopping with scripted random draws, rescaling, decoherence, centre of mass and
rotation) on stand-in objects, through the same shim.

Usage::

    python tests/golden/make_golden.py /path/to/DFTBaby [--only=core|couplings|mulliken|sk_python|scc|lr_glue|lambda|repulsive|lr_e2e|particle_hole|handler|dftb2_props|xyz|md|initial_conditions]
"""
import io
import os
import re
import shutil
import sys
import tempfile
import tokenize
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def py2to3(src):
    """Mechanical conversion of print statements and renamed dict/range methods."""
    src = src.replace(".iteritems()", ".items()").replace("xrange(", "range(")
    src = re.sub(r"\.has_key\(", ".__contains__(", src)
    src = src.replace(".translate(None, digits)", ".translate(str.maketrans('', '', digits))")
    # one-line "print>>fh, a, b" statements -> print(a, b, file=fh); a trailing comma keeps the line open
    # (end=" " writes the space Python 2's softspace would write before the next item on that line)
    src = re.sub(r"^(\s*)print\s*>>\s*([^,\n]+),\s*(.*?),\s*$", r'\1print(\3, end=" ", file=\2)', src, flags=re.M)
    src = re.sub(r"^(\s*)print\s*>>\s*([^,\n]+),\s*(.*)$", r"\1print(\3, file=\2)", src, flags=re.M)
    toks = list(tokenize.generate_tokens(io.StringIO(src).readline))
    edits = []
    for k, t in enumerate(toks):
        if t.type != tokenize.NAME or t.string != "print":
            continue
        j = k - 1
        while j >= 0 and toks[j].type in (tokenize.NL, tokenize.COMMENT):
            j -= 1
        if j >= 0 and toks[j].type not in (tokenize.NEWLINE, tokenize.INDENT, tokenize.DEDENT) \
                and toks[j].string != ":":
            continue
        if toks[k + 1].string == "(" and toks[k + 1].start[1] == t.end[1]:
            continue  # already a call (converted above)
        m = k + 1
        while toks[m].type not in (tokenize.NEWLINE, tokenize.ENDMARKER):
            m += 1
        e = m - 1
        while toks[e].type in (tokenize.COMMENT, tokenize.NL):
            e -= 1
        if e == k:
            edits.append((t.start, t.end, "print()"))
        elif toks[e].string == ",":
            edits.append((toks[e].start, toks[e].end, ', end=" ")'))
            edits.append((t.start, t.end, "print("))
        else:
            edits.append((toks[e].end, toks[e].end, ")"))
            edits.append((t.start, t.end, "print("))
    lines = src.splitlines(keepends=True)
    for (r0, c0), (r1, c1), text in sorted(edits, key=lambda x: (x[0], x[1]), reverse=True):
        assert r0 == r1
        ln = lines[r0 - 1]
        lines[r0 - 1] = ln[:c0] + text + ln[c1:]
    return "".join(lines)


def load_reference_modules(ref_root):
    """Build a temporary ``DFTB`` package holding shimmed copies of the needed modules."""
    tmp = tempfile.mkdtemp(prefix="dftbaby_ref_")
    pkg = os.path.join(tmp, "DFTB")
    os.makedirs(os.path.join(pkg, "extensions"))
    open(os.path.join(pkg, "__init__.py"), "w").close()
    open(os.path.join(pkg, "extensions", "__init__.py"), "w").write("tddftb = None\nslako = None\ngrad = None\n")
    os.makedirs(os.path.join(pkg, "SlaterKoster"))
    open(os.path.join(pkg, "SlaterKoster", "__init__.py"), "w").close()
    open(os.path.join(pkg, "SlaterKoster", "SKIntegrals.py"), "w").write("combine_slako_tables_f90 = None\n")
    open(os.path.join(pkg, "SKMatrixElements.py"), "w").write(
        "SLAKO_IMPLEMENTATION = 'PY'\natomlist2orbitals = None\n")
    open(os.path.join(pkg, "DiskMemory.py"), "w").write(
        "class _M:\n    def memmap(self, f):\n        return f\nGlobalDiskMemory = _M()\n")
    for stub in ("XYZ", "utils", "CPKS"):
        open(os.path.join(pkg, stub + ".py"), "w").close()
    open(os.path.join(pkg, "Timer.py"), "w").write(
        "class _T:\n    def timer(self, f):\n        return f\nGlobalTimer = _T()\n")
    open(os.path.join(pkg, "AtomicData.py"), "w").write("atom_names = ['h','he','li','be','b','c']\n")
    names = ("Solver", "GammaApproximation", "ConvAcceleration", "ExcGradients")
    for name in names:
        src = open(os.path.join(ref_root, "DFTB", name + ".py")).read()
        open(os.path.join(pkg, name + ".py"), "w").write(py2to3(src))
    sys.path.insert(0, tmp)
    import importlib
    mods = {n: importlib.import_module("DFTB." + n) for n in names}
    return tmp, mods


def sk_rule_cases(ref_root):
    """Parse the reference's SK rule tables: {(l1,m1,l2,m2): expr} and {(l1,m1,mr,l2,m2): expr}."""
    ext = os.path.join(ref_root, "DFTB", "extensions")
    pat = re.compile(r"CASE \((\d+)\)\s*\n\s*! \(([^)]*)\)\s*\n\s*res = ([^\n]*)")
    sh = {}
    for _, tup, expr in pat.findall(open(os.path.join(ext, "slako_transformations_lmax2.f90")).read()):
        key = tuple(int(v) for v in tup.split(","))
        if key[0] <= 1 and key[2] <= 1:
            sh[key] = expr
    dip = {}
    for _, tup, expr in pat.findall(open(os.path.join(ext, "slako_transformations_dipole_lmax2.f90")).read()):
        key = tuple(int(v) for v in tup.split(","))
        if key[0] <= 1 and key[3] <= 1:
            dip[key] = expr
    return sh, dip


def make_sk_rules(ref_root, rng):
    sh, dip = sk_rule_cases(ref_root)
    ndir = 16
    e = rng.normal(size=(ndir, 3))
    e /= np.linalg.norm(e, axis=1)[:, None]
    V = rng.normal(size=(ndir, 7))
    Dt = rng.normal(size=(ndir, 15))
    sh_keys = np.array(sorted(sh), dtype=np.int64)
    dip_keys = np.array(sorted(dip), dtype=np.int64)
    sh_val = np.zeros((ndir, len(sh_keys)))
    dip_val = np.zeros((ndir, len(dip_keys)))
    for n in range(ndir):
        env = dict(x=e[n, 0], y=e[n, 1], z=e[n, 2], sqrt3=np.sqrt(3.0))
        env["SorH"] = lambda k, n=n: V[n, k - 1]
        env["Dip"] = lambda k, n=n: Dt[n, k - 1]
        for c, key in enumerate(sh_keys):
            sh_val[n, c] = eval(sh[tuple(key)], env)
        for c, key in enumerate(dip_keys):
            dip_val[n, c] = eval(dip[tuple(key)], env)
    np.savez_compressed(os.path.join(HERE, "sk_rules.npz"), e=e, V=V, D=Dt, sh_keys=sh_keys, sh_val=sh_val,
                        dip_keys=dip_keys, dip_val=dip_val)


def sk_grad_rule_cases(ref_root):
    """{(l1,m1,l2,m2): {c: expr}} from slako_transformations_grad_lmax2.f90 (s and p only)."""
    src = open(os.path.join(ref_root, "DFTB", "extensions", "slako_transformations_grad_lmax2.f90")).read()
    src = re.sub(r"&\s*\n\s*&?", "", src)   # join Fortran continuation lines
    pat = re.compile(r"CASE \((\d+)\)\s*\n\s*! \(([^)]*)\)\s*\n\s*grad\((\d)\) = ([^\n]*)")
    cases = {}
    for _, tup, c, expr in pat.findall(src):
        key = tuple(int(v) for v in tup.split(","))
        if key[0] <= 1 and key[2] <= 1:
            cases.setdefault(key, {})[int(c) - 1] = expr
    return cases


def make_sk_grad_rules(ref_root, rng):
    cases = sk_grad_rule_cases(ref_root)
    ndir = 16
    e = rng.normal(size=(ndir, 3))
    e /= np.linalg.norm(e, axis=1)[:, None]
    r = rng.uniform(1.0, 8.0, size=ndir)
    V = rng.normal(size=(ndir, 7))
    Vd = rng.normal(size=(ndir, 7))
    keys = np.array(sorted(cases), dtype=np.int64)
    val = np.zeros((ndir, len(keys), 3))
    for n in range(ndir):
        env = dict(x=e[n, 0], y=e[n, 1], z=e[n, 2], r=r[n], sqrt3=np.sqrt(3.0))
        env["SorH"] = lambda k, n=n: V[n, k - 1]
        env["SorHd"] = lambda k, n=n: Vd[n, k - 1]
        for j, key in enumerate(keys):
            for c in range(3):
                val[n, j, c] = eval(cases[tuple(key)][c], env)
    np.savez_compressed(os.path.join(HERE, "sk_grad_rules.npz"), e=e, r=r, V=V, Vd=Vd, keys=keys, val=val)


def make_gradients(mods, rng):
    """DFTBaby's ExcGradients.Gradients.gradient on a seeded C4H6, lc on and off, states 0, 1, 2."""
    EG, GA = mods["ExcGradients"], mods["GammaApproximation"]
    sys.path.insert(0, REPO)
    from dftbaby_b200 import geometry
    from oracle import dftb_oracle as O
    from oracle import gradients_oracle as G

    class _Vrep:
        def __init__(self, par, Z1, Z2):
            self.par, self.Z1, self.Z2 = par, Z1, Z2

        def getVrep(self, R, deriv=0):
            return self.par.getVrep(self.Z1, self.Z2, R, deriv)

    al = geometry.polyene(4, sigma=0.05, seed=7)
    out = {"Z": np.array([z for z, _ in al]), "pos": np.array([p for _, p in al])}
    for lc in (1, 0):
        td = O.LR_TDDFTB(al, long_range_correction=lc)
        td.setGeometry(al)
        td.getEnergies(nstates=4, diag_conv=1.0e-10, diag_maxiter=200)
        d = td.dftb2
        gS, gH = G.gradients_H0andS(d)
        EG.gradients_H0andS = lambda *a, **k: (gS, gH)
        fd = types.SimpleNamespace()
        fd.atomlist = d.atomlist
        fd.getGeometry = lambda: d.atomlist
        fd.valorbs = d.valorbs
        fd.distances, fd.directions = d.distances, d.directions
        sig = GA.gaussian_decay(d.par.hubbard_U, d.valorbs, d.long_range_radius, lc, verbose=0)
        fd.gm = GA.GammaMatrix(GA.GammaGaussian(sig))
        fd.gm_lc = GA.GammaMatrix(GA.GammaGaussianLC(sig, d.long_range_radius))
        fd.getKSEnergies, fd.getKSCoefficients = (lambda: d.orbe), (lambda: d.orbs)
        fd.verbose, fd.SKT, fd.Mproximity, fd.S = 0, None, d.Mproximity, d.S
        fd.density_matrix_ref = d.density_matrix_ref
        fd.lc_implementation, fd.long_range_correction = None, lc
        fd.VREP = {(a, b): _Vrep(d.par, a, b) for (a, b) in d.par.vrep}
        ft = types.SimpleNamespace(dftb2=fd, ct_correction=0)
        ft.getActiveOrbitals = lambda: (td.active_occupied_orbs, td.active_virtual_orbs)
        ft.hasActiveSpace = lambda: False
        ft.getXY = lambda: (td.XmY, td.XpY)
        ft.getExcEnergies = lambda: td.Omega
        ft.getTransitionCharges = lambda: (td.qtrans_oo, td.qtrans_vv, td.qtrans_ov)
        grads = EG.Gradients(ft)
        for I in (0, 1, 2):
            gV, gE, gX = grads.gradient(I=I)
            tag = "lc%d_I%d" % (lc, I)
            out[tag + "_Vrep"], out[tag + "_E0"], out[tag + "_Exc"] = gV, gE, gX
        out["lc%d_Omega" % lc] = td.Omega
    np.savez_compressed(os.path.join(HERE, "gradients_c4h6.npz"), **out)


def make_gamma(mods, rng):
    GA = mods["GammaApproximation"]
    from dftbaby_b200 import geometry
    al = geometry.polyene(6, sigma=0.05, seed=3)
    hub = {1: (13.5984 - 0.75419) / 27.211396132, 6: (11.2603 - 1.262119) / 27.211396132}
    valorbs = {1: [(0, 0, 0)], 6: [(1, 0, 0), (1, 1, -1), (1, 1, 0), (1, 1, 1)]}
    sig = GA.gaussian_decay(hub, valorbs, 3.03, 1, verbose=0)
    pos = np.array([p for _, p in al])
    R = pos[:, None] - pos[None]
    dist = np.sqrt(np.sum(R * R, axis=-1))
    nat = len(al)
    dirs = np.zeros((nat, nat, 3))
    off = dist > 0
    dirs[off] = R[off] / dist[off][:, None]
    g = GA.GammaMatrix(GA.GammaGaussian(sig)).gamma_atomwise(al, dist)[0]
    glr, _, Glr, _ = GA.GammaMatrix(GA.GammaGaussianLC(sig, 3.03)).gamma_AOwise(al, valorbs, dist, dirs)
    np.savez_compressed(os.path.join(HERE, "gamma.npz"), Z=np.array([z for z, _ in al]), pos=pos,
                        sigma_H=sig[1], sigma_C=sig[6], gamma=g, gamma_lr=glr, G_lr=Glr)


def make_diis(mods, rng):
    CA = mods["ConvAcceleration"]
    n = 12
    A = rng.normal(size=(n, n)) * 0.15
    b = rng.normal(size=n)
    x = np.zeros(n)
    mixer = CA.DIIS_80(5)
    xs_in, xs_out, rel = [], [], []
    for it in range(25):
        x_new = np.dot(A, x) + b
        xs_in.append(x_new.copy())
        x = mixer.next_approximation(x_new.copy())
        xs_out.append(np.array(x, dtype=float).copy())
        rel.append(mixer.relative_change())
    np.savez_compressed(os.path.join(HERE, "diis.npz"), A=A, b=b, xs_in=np.array(xs_in),
                        xs_out=np.array(xs_out), rel=np.array(rel))


def make_solvers(mods, rng):
    """Reference solvers on transition charges of a seeded C10H12 (lc on)."""
    SV = mods["Solver"]
    sys.path.insert(0, REPO)
    from dftbaby_b200 import geometry
    from oracle import dftb_oracle as O
    al = geometry.polyene(10, sigma=0.02, seed=0)
    td = O.LR_TDDFTB(al, long_range_correction=1)
    td.setGeometry(al)
    td.dftb2.getEnergy()
    td.setActiveOrbitals(None, None)
    d = td.dftb2
    co, cv = d.orbs[:, td.active_occupied_orbs], d.orbs[:, td.active_virtual_orbs]
    q_oo, q_ov, q_vv = O.trans_charges(co, cv, d.S, d.orbsPerAtom)
    no, nv = td.nocc, td.nvirt
    orbe = d.orbe
    omega = orbe[td.active_virtual_orbs][None, :] - orbe[td.active_occupied_orbs][:, None]
    df = np.full((no, nv), 2.0)
    shift = np.zeros((no, nv))
    g, glr = d.gamma, d.gamma_lr
    out = dict(q_oo=q_oo, q_ov=q_ov, q_vv=q_vv, omega=omega, gamma=g, gamma_lr=glr)
    for tag, gl in (("lc", glr), ("nolc", 0.0 * glr)):
        Om, C, XmY, XpY = SV.Casida(g, gl, q_oo, q_vv, q_ov, omega, shift, df, no, nv)
        out["casida_%s_Omega" % tag] = Om
        out["casida_%s_XmY" % tag] = XmY[:8]
        out["casida_%s_XpY" % tag] = XpY[:8]
    Oia = np.zeros((no, nv))
    Om, C, XmY, XpY = SV.HermitianDavidson(g, q_ov, omega, shift, no, nv, None, None, Oia, nstates=6, ifact=1,
                                           conv=1.0e-9, maxiter=100, L2_thresh=0.0, verbose=0)
    out.update(herm_Omega=Om, herm_C=C, herm_XmY=XmY, herm_XpY=XpY)
    Om, C, XmY, XpY = SV.nonHermitianDavidson(g, glr, q_oo, q_vv, q_ov, omega, no, nv, None, None, None,
                                              nstates=6, ifact=1, conv=1.0e-9, maxiter=100, verbose=0, lc=1)
    out.update(nonherm_Omega=Om, nonherm_C=C, nonherm_XmY=XmY, nonherm_XpY=XpY)
    vs = rng.normal(size=(no, nv, 3))
    out["vs"] = vs
    out["ApBv"] = SV._ApBv(g, glr, q_oo, q_ov, q_vv, omega, vs, 1)
    out["AmBv"] = SV._AmBv(g, glr, q_oo, q_ov, q_vv, omega, vs, 1)
    np.savez_compressed(os.path.join(HERE, "solvers_c10h12.npz"), **out)


def method_source(path, name, after=None):
    """The text of method ``name`` of a DFTBaby source file, dedented and passed through the shim.
    Tabs are expanded to 8 columns (Python 2's rule for mixed indentation) and ``<>`` becomes ``!=``.
    With ``after`` (a regular expression) the search starts at the first line matching it."""
    lines = open(path).read().expandtabs(8).splitlines(keepends=True)
    first = 0 if after is None else next(i for i, ln in enumerate(lines) if re.match(after, ln))
    start = next(i for i in range(first, len(lines)) if re.match(r"\s*def %s\(" % name, lines[i]))
    indent = len(lines[start]) - len(lines[start].lstrip())
    end = start + 1
    in_string = False  # inside a triple-quoted string, whose lines may start at any column
    body = [lines[start]]
    while end < len(lines):
        ln = lines[end]
        if not in_string and ln.strip() and not ln.lstrip().startswith("#") and len(ln) - len(ln.lstrip()) <= indent:
            break
        # comment lines indented less than the def (trailing section headers) are not part of the method
        if in_string or not (ln.lstrip().startswith("#") and len(ln) - len(ln.lstrip()) < indent):
            body.append(ln)
        if (ln.count('"""') + ln.count("\'\'\'")) % 2 == 1:
            in_string = not in_string
        end += 1
    # remove the def's indentation from every line that has it (string lines may have less)
    text = "".join(ln[indent:] if ln[:indent].strip() == "" else ln for ln in body)
    return py2to3(text.replace("<>", "!="))


def _reference_methods(path, names, namespace):
    ns = dict(namespace)
    for n in names:
        exec(compile(method_source(path, n), "%s:%s" % (os.path.basename(path), n), "exec"), ns)
    return ns


def make_couplings(ref_root, rng):
    """ScalarCoupling.ci_overlap (AO overlap supplied), PES.getScalarCouplings (phase alignment) and the
    electronic and nuclear steps of SurfaceHopping.MolecularDynamics, run from DFTBaby's own method
    texts on synthetic inputs."""
    import numpy.linalg as la
    import scipy.linalg as sla
    out = {}
    # ---- CI overlaps: 16 orbitals, 6 doubly occupied, active occ 2..5, virt 6..10
    norb, nelec, occ, virt, nst = 16, 12, np.arange(2, 6), np.arange(6, 11), 5
    Q1, _ = np.linalg.qr(rng.standard_normal((norb, norb)))
    Q2, _ = np.linalg.qr(Q1 + 0.1 * rng.standard_normal((norb, norb)))
    Sao = np.eye(norb) + 0.05 * rng.standard_normal((norb, norb))
    C1 = 0.5 * rng.standard_normal((nst, len(occ), len(virt)))
    C2 = 0.5 * rng.standard_normal((nst, len(occ), len(virt)))
    C1[:, 1, 2] = 4e-3
    C2[:, 0, 4] = -2e-3
    ns = _reference_methods(os.path.join(ref_root, "DFTB", "ScalarCoupling.py"), ["ci_overlap"],
                            {"np": np, "la": la, "overlap_AB": lambda *a: Sao})

    class _D:
        verbose, qmmm, valorbs, SKT, Nelec_val = 0, None, None, None, nelec

    class _TD:
        dftb2 = _D()

        def getActiveOrbitals(self):
            return occ, virt

    sc = types.SimpleNamespace(tddftb=_TD())
    for k, thr in enumerate((1e-3, 1e-2)):
        out["sci_%d" % k] = ns["ci_overlap"](sc, None, Q1, C1, None, Q2, C2, nst + 1, threshold=thr)
    out.update(sao=Sao, orbs1=Q1, orbs2=Q2, C1=C1, C2=C2, nelec=nelec, occ=occ, virt=virt,
               thresholds=np.array([1e-3, 1e-2]))
    # ---- phase alignment over two calls (PES.py:180-252)
    Sci_steps = []
    for step in range(2):
        A = 0.05 * rng.standard_normal((4, 4))
        S = np.eye(4) + A - A.T + 0.01 * rng.standard_normal((4, 4))
        S = S @ np.diag([1.0, -1.0, 1.0, -1.0] if step == 0 else [1.0, 1.0, -1.0, -1.0])
        if step == 1:
            S[0, 1:] *= -1.0
            S[1:, 0] *= -1.0
        Sci_steps.append(S)
    Cj = [rng.standard_normal((3, 2, 3)) for _ in range(2)]
    it = iter(Sci_steps)

    class _SC:
        def __init__(self, td):
            pass

        def ci_overlap(self, *args, **kw):
            return next(it)

    ns = _reference_methods(os.path.join(ref_root, "DFTB", "PES.py"), ["getScalarCouplings"],
                            {"np": np, "ScalarCoupling": _SC, "utils": None})
    pes = types.SimpleNamespace(atomlist=None, Nst=4, last_calculation=None,
                                tddftb=types.SimpleNamespace(dftb2=types.SimpleNamespace(orbs=None, verbose=0)))
    for step in range(2):
        pes.tddftb.Cij = Cj[step]
        coupl, olap = ns["getScalarCouplings"](pes, threshold=0.01)
        out["pes_sci_%d" % step] = Sci_steps[step]
        out["pes_C_%d" % step] = Cj[step]
        out["pes_coupl_%d" % step], out["pes_olap_%d" % step] = coupl, olap
        out["pes_P_%d" % step] = pes.P
        out["pes_C_aligned_%d" % step] = pes.last_calculation[2]
    # ---- surface hopping steps (SurfaceHopping.py:149-201, 262-399)
    sh_path = os.path.join(ref_root, "DFTB", "Dynamics", "SurfaceHopping.py")
    draws = iter([0.05, 0.1, 0.6])
    ns = _reference_methods(sh_path, ["getLocalDiabatization", "getNewState", "getUniformlyRescaledVelocities",
                                      "getDecoherenceE", "getCenterOfMass", "shiftToCenterOfMass", "momentum",
                                      "eliminateTranslation", "myCrossProduct", "angularMomentum",
                                      "momentOfInertia", "getAngularVelocity", "eliminateRotation",
                                      "eliminateTransRot", "getKineticEnergy"],
                            {"np": np, "la": la, "sla": sla,
                             "random": types.SimpleNamespace(random=lambda: next(draws))})

    class _MD:
        pass

    for name in [k for k in ns if callable(ns[k]) and not k.startswith("_") and k[0].islower()]:
        if name in ("random",):
            continue
        setattr(_MD, name, ns[name])
    md = _MD()
    nat = 5
    md.masses = np.array([12.0, 12.0, 1.0, 1.0, 16.0]) * 1822.888
    md.totalmass = md.masses.sum()
    md.coordinates = rng.standard_normal((nat, 3)) * 2.0
    md.velocities = rng.standard_normal((nat, 3)) * 1e-3
    md.nat = nat
    md.printcoeff = 0
    md.switch_to_groundstate = 1
    md.decoherence_constant = 0.1
    md.tstep = 20.0
    md.time = 0.0
    md.au_to_fs = 0.0241888
    md.nstates = 4
    A = 0.08 * rng.standard_normal((4, 4))
    md.olap = sla.expm(A - A.T)
    md.energy_last = np.array([-10.0, -9.85, -9.80, -9.70])
    md.energy = np.array([-10.001, -9.845, -9.815, -9.69])
    md.c = np.array([0.1, 0.9, 0.3 + 0.2j, 0.2j], dtype=complex)
    md.c /= np.linalg.norm(md.c)
    out.update(sh_olap=md.olap, sh_E0=md.energy_last, sh_E1=md.energy, sh_c0=md.c.copy(), sh_dt=md.tstep)
    md.getLocalDiabatization()
    out["sh_c1"] = md.c.copy()
    # hops: flux out of state 1 into 2 and 3, three scripted draws
    c_old = np.sqrt(np.array([0.0, 0.9, 0.06, 0.04])).astype(complex)
    c_new = np.sqrt(np.array([0.0, 0.8, 0.12, 0.08])).astype(complex)
    states = []
    for _ in range(3):
        md.state, md.c_old, md.c = 1, c_old.copy(), c_new.copy()
        md.getNewState()
        states.append(md.state)
    out.update(hop_c_old=c_old, hop_c=c_new, hop_draws=np.array([0.05, 0.1, 0.6]), hop_states=np.array(states))
    # rescaling and decoherence
    md.kinetic_energy = md.getKineticEnergy(md.velocities, md.masses)
    v0 = md.velocities.copy()
    md.state, md.oldstate = 2, 1
    md.getUniformlyRescaledVelocities()
    out.update(res_v0=v0, res_ekin=md.kinetic_energy, res_state=md.state, res_v=md.velocities.copy())
    md.velocities = v0.copy()
    md.energy = np.array([-10.0, -9.9, -9.9 + 3 * md.kinetic_energy, -9.7])
    md.state, md.oldstate = 2, 1
    md.getUniformlyRescaledVelocities()
    out.update(rej_E=md.energy.copy(), rej_state=md.state, rej_v=md.velocities.copy())
    md.energy = np.array([-10.001, -9.845, -9.815, -9.69])
    md.c = out["sh_c0"].copy()
    md.state = 1
    md.getDecoherenceE()
    out["dec_c"] = md.c.copy()
    # centre of mass, translation and rotation
    x0, v0 = md.coordinates.copy(), md.velocities.copy()
    md.coordinates = md.shiftToCenterOfMass(md.coordinates)
    md.velocities = v0.copy()
    md.eliminateTransRot()
    out.update(com_x0=x0, com_x=md.coordinates.copy(), com_v0=v0, com_v=md.velocities.copy(), com_m=md.masses)
    np.savez_compressed(os.path.join(HERE, "couplings.npz"), **out)


def make_mulliken_trans_charges(ref_root, rng):
    """Mulliken.monopoles (Mulliken.py:10-48, the Python twin of mulliken.f90) and the Python loop of
    LR_TDDFTB._MullikenTransitionCharges (LR_TDDFTB.py:267-296, the twin of tddftb.trans_charges,
    which the reference keeps in a string next to the Fortran call), on a C4H6 orbital layout."""
    import textwrap
    Zs = [6, 6, 6, 6, 1, 1, 1, 1, 1, 1]
    valorbs = {1: [(1, 0, 0)], 6: [(2, 0, 0), (2, 1, -1), (2, 1, 0), (2, 1, 1)]}
    atomlist = [(Z, (0.0, 0.0, float(k))) for k, Z in enumerate(Zs)]
    norb = sum(len(valorbs[Z]) for Z in Zs)
    X = rng.standard_normal((norb, norb))
    S = np.eye(norb) + 0.1 * (X + X.T)
    X = rng.standard_normal((norb, norb))
    P = 0.5 * (X + X.T)
    P0 = np.diag(rng.random(norb))
    ns = {"np": np}
    exec(compile(method_source(os.path.join(ref_root, "DFTB", "Mulliken.py"), "monopoles"), "Mulliken.py", "exec"),
         ns)
    q, dq = ns["monopoles"](atomlist, P, P0, S, valorbs)
    # the Python block of _MullikenTransitionCharges, between "# PYTHON CODE" and the closing quotes
    lines = open(os.path.join(ref_root, "DFTB", "LR_TDDFTB.py")).read().expandtabs(8).splitlines(keepends=True)
    start = next(i for i, ln in enumerate(lines) if ln.strip() == "# PYTHON CODE")
    end = next(i for i in range(start + 1, len(lines)) if lines[i].strip() == '"""')
    block = py2to3(textwrap.dedent("".join(lines[start:end])))
    orbs = np.linalg.qr(rng.standard_normal((norb, norb)))[0]
    occ, virt = np.array([3, 5, 6, 7, 8]), np.array([11, 12, 14, 20])
    fake = types.SimpleNamespace(active_occupied_orbs=occ, active_virtual_orbs=virt)
    ns = {"zeros": np.zeros, "dot": np.dot, "self": fake, "atomlist": atomlist, "valorbs": valorbs,
          "orbs": orbs, "S": S}
    exec(compile(block, "LR_TDDFTB.py:_MullikenTransitionCharges", "exec"), ns)
    np.savez_compressed(os.path.join(HERE, "mulliken_trans_charges.npz"), Z=np.array(Zs), S=S, P=P, P0=P0,
                        q=q, dq=dq, orbs=orbs, occ=occ, virt=virt, q_oo=fake.qtrans_oo, q_ov=fake.qtrans_ov,
                        q_vv=fake.qtrans_vv)


def make_sk_python(ref_root, rng):
    """S, H0, D and the gradients of S and H0 from DFTBaby's Python Slater-Koster path:
    SKMatrixElements._H0andS and _DipoleMatrix (SKMatrixElements.py:64-131, 263-318) and
    ExcGradients._gradients_H0andS (ExcGradients.py:52-141) over SlakoTransformations (SKIntegrals.py:832-1070), whose splines are splrep(s=None) fits of the
    shipped tables (spline_slako_integrals, SKIntegrals.py:793-827) evaluated exactly, with the Python
    angular rules of slako_transformations.py.  Two compact geometries (all pairs inside the 10-bohr
    tables), every pair interacting."""
    from scipy import interpolate

    sys.path.insert(0, REPO)
    from oracle import dftb_oracle as O
    sk = os.path.join(ref_root, "DFTB", "SlaterKoster")

    def load(path, shim):
        src = open(path).read()
        if shim:
            src = py2to3(src.expandtabs(8))
        mod = types.ModuleType(os.path.basename(path)[:-3])
        exec(compile(src, path, "exec"), mod.__dict__)
        return mod

    T = load(os.path.join(sk, "slako_transformations.py"), True)
    Tdip = load(os.path.join(sk, "slako_transformations_dipole.py"), True)
    tables = {key: load(os.path.join(sk, "slako_tables", name + ".py"), False)
              for key, name in (((1, 1), "h_h"), ((1, 6), "h_c"), ((6, 6), "c_c"))}
    ns = {"np": np, "interpolate": interpolate, "T": T, "Tdip": Tdip, "sqrt": np.sqrt, "reshape": np.reshape,
          "where": np.where, "zeros": np.zeros, "AtomicData": None, "NoSKDipolesException": RuntimeError}
    ski = os.path.join(sk, "SKIntegrals.py")
    exec(compile(method_source(ski, "spline_slako_integrals"), "SKIntegrals.py", "exec"), ns)
    names = ("__init__", "_directional_cosines", "getOverlap", "getHamiltonian0", "haveDipoles", "getDipole")
    for n in names:
        exec(compile(method_source(ski, n, after=r"class SlakoTransformations"), "SKIntegrals.py", "exec"), ns)
    ST = type("SlakoTransformations", (), {n: ns[n] for n in names})
    SKT = {key: ST(mod) for key, mod in tables.items()}
    skm = os.path.join(ref_root, "DFTB", "SKMatrixElements.py")
    ns2 = {"np": np}
    for n in ("count_orbitals", "_H0andS", "_DipoleMatrix"):
        exec(compile(method_source(skm, n), "SKMatrixElements.py", "exec"), ns2)
    ns3 = {"np": np}
    exec(compile(method_source(os.path.join(ref_root, "DFTB", "ExcGradients.py"), "_gradients_H0andS"),
                 "ExcGradients.py", "exec"), ns3)
    par = O.Parametrization([1, 6])
    out = {}
    geoms = []
    from dftbaby_b200 import geometry
    geoms.append(geometry.polyene(2, sigma=0.05, seed=3))  # C2H4
    while True:  # a random C3H3 cluster, all pairs 1.8-9 bohr apart
        pos = rng.uniform(-3.0, 3.0, size=(6, 3))
        d = np.linalg.norm(pos[:, None] - pos[None], axis=-1)[np.triu_indices(6, 1)]
        if d.min() > 1.8 and d.max() < 9.0:
            break
    geoms.append([(Z, tuple(p)) for Z, p in zip([6, 1, 6, 1, 6, 1], pos)])
    for k, al in enumerate(geoms):
        nat = len(al)
        S, H0 = ns2["_H0andS"](al, al, par.valorbs, SKT, par.orbital_energies, np.ones((nat, nat), dtype=int))
        out["Z_%d" % k] = np.array([Z for Z, _ in al])
        out["pos_%d" % k] = np.array([p for _, p in al])
        out["S_%d" % k], out["H0_%d" % k] = S, H0
        out["D_%d" % k] = ns2["_DipoleMatrix"](al, al, par.valorbs, SKT, np.ones((nat, nat), dtype=int))
        out["gradS_%d" % k], out["gradH0_%d" % k] = ns3["_gradients_H0andS"](al, par.valorbs, SKT,
                                                                              np.ones((nat, nat), dtype=int))
    np.savez_compressed(os.path.join(HERE, "sk_python.npz"), **out)


def _twisted_ethylene():
    """C2H4 twisted by 90 degrees about the C=C bond (bohr): HOMO and LUMO nearly degenerate."""
    cc, ch, a = 2.53, 2.05, np.deg2rad(121.0)
    hx, hr = ch * np.cos(np.pi - a), ch * np.sin(np.pi - a)
    return [(6, (0.0, 0.0, 0.0)), (6, (cc, 0.0, 0.0)),
            (1, (-hx, hr, 0.0)), (1, (-hx, -hr, 0.0)),
            (1, (cc + hx, 0.0, hr)), (1, (cc + hx, 0.0, -hr))]


def _reference_dftb2(ref_root, mods):
    """A DFTB2 stand-in class carrying DFTBaby's own runSCC and its helpers (DFTB2.py:702-717, 804-879,
    940-1160, 1239-1266, 2516-2610, and the frontier-orbital accessors), run from their text.  Mulliken
    charges come from the oracle's restatement of mulliken.f90 (pinned against Mulliken.monopoles); the
    energies, which the iteration does not use, are skipped."""
    import scipy.linalg as sla

    sys.path.insert(0, REPO)
    from oracle import dftb_oracle as O

    class SCFNotConverged(Exception):
        pass

    class SCFChargeInconsistency(Exception):
        pass

    dftb2 = os.path.join(ref_root, "DFTB", "DFTB2.py")
    mull = types.SimpleNamespace(mulliken=types.SimpleNamespace(
        monopoles=lambda P, P0, S, opa: O.monopoles(P, P0, S, np.asarray(opa, dtype=np.int32))))
    ns = {"np": np, "la": np.linalg, "array": np.array, "zeros": np.zeros, "sqrt": np.sqrt, "log": np.log,
          "exp": np.exp, "dot": np.dot, "argsort": np.argsort, "where": np.where, "sum": np.sum,
          "eigh": sla.eigh, "norm": sla.norm, "inv": sla.inv, "sqrtm": sla.sqrtm, "copy": np.copy,
          "DIIS_80": mods["ConvAcceleration"].DIIS_80, "mulliken": mull, "SCFNotConverged": SCFNotConverged,
          "SCFChargeInconsistency": SCFChargeInconsistency, "kBoltzmann": 3.166811382e-6}
    for n in ("fermi_occupation", "fermi_occupation_T0"):
        exec(compile(method_source(dftb2, n), "DFTB2.py", "exec"), ns)
    names = ("runSCC", "_coulomb_hamiltonian", "_construct_h1", "lc_exact_exchange", "density_matrix_ref",
             "_constructDensityMatrix", "_density_matrix", "_MullikenAnalysis", "getHOMO_LUMO_gap",
             "getFrontierOrbitals")
    for n in names:
        exec(compile(method_source(dftb2, n, after=r"class DFTB2"), "DFTB2.py", "exec"), ns)
    return type("DFTB2", (), dict({n: ns[n] for n in names}, getEnergies=lambda self: None))


def _load_into(ref, od, lc):
    """Copy the oracle's matrices for one geometry into a reference DFTB2 stand-in."""
    ref.atomlist, ref.valorbs, ref.valorbs_occupation = od.atomlist, od.par.valorbs, od.par.valorbs_occupation
    ref.dim, ref.S, ref.H0, ref.gamma = od.dim, od.S, od.H0, od.gamma
    ref.G_lr = od.G_lr if lc else None
    ref.gamma_lr = od.gamma_lr if lc else None
    ref.long_range_correction, ref.lc_implementation = lc, "new"
    ref.Nelec_val, ref.nr_unpaired_electrons, ref.charge = od.Nelec_val, 0, 0.0
    ref.orbsPerAtom, ref.charge_guess, ref.verbose = od.orbsPerAtom, None, 0
    ref.mulliken_dipoles, ref.point_charges, ref.onsite_correction, ref.save_converged_charges = 0, [], 0, None


def make_scc(ref_root, mods):
    """DFTB2.runSCC (DFTB2.py:940-1160) with its helpers run from DFTBaby's text (``_reference_dftb2``) on
    the oracle's S, H0, gamma and G_lr, with the default DIIS_80 mixer of the shimmed ConvAcceleration.
    Three cases: C10H12 with the long-range correction, C6H8 without, and a 90-degree twisted ethylene
    whose near-degenerate frontier orbitals switch the level shift on."""
    from dftbaby_b200 import geometry
    from oracle import dftb_oracle as O
    Ref = _reference_dftb2(ref_root, mods)
    out = {}
    cases = (("c10h12_lc", geometry.polyene(10, sigma=0.02, seed=11), 1),
             ("c6h8", geometry.polyene(6, sigma=0.02, seed=12), 0),
             ("twisted_c2h4_lc", _twisted_ethylene(), 1))
    for name, al, lc in cases:
        od = O.DFTB2(al, long_range_correction=lc)
        od.setGeometry(al)
        od.getEnergy()  # builds the oracle's matrices (and runs its own SCC, not used here)
        r = Ref()
        _load_into(r, od, lc)
        r.runSCC()
        out["%s_Z" % name] = np.array([Z for Z, _ in al])
        out["%s_pos" % name] = np.array([p for _, p in al])
        out["%s_lc" % name] = lc
        out["%s_iterations" % name] = r.i + 1
        for key in ("P", "dq", "orbe", "f", "HLgap", "relative_change", "S", "H0"):
            out["%s_%s" % (name, key)] = getattr(r, key)
    np.savez_compressed(os.path.join(HERE, "scc.npz"), **out)


def make_lr_glue(ref_root, rng):
    """LR_TDDFTB.setActiveOrbitals, setActiveLMOrbitals, _TransitionDipoles, _TransitionDipolesMulliken, getTransitionDipolesExc,
    getOscillatorStrengths, determineActiveSpace, TransitionChargesState, saveAbsorptionSpectrum,
    saveTransitionCharges, _dominant_excitations and _writeExcitations (LR_TDDFTB.py:125-243, 567-831, 900-908,
    1008-1025) run from DFTBaby's text on a
    stand-in solved object: 14 orbitals (6 doubly occupied), active window 3 x 4, 3 states."""
    lr = os.path.join(ref_root, "DFTB", "LR_TDDFTB.py")
    names = ("setActiveOrbitals", "_TransitionDipoles", "_TransitionDipolesMulliken", "getOscillatorStrengths",
             "determineActiveSpace", "TransitionChargesState", "saveAbsorptionSpectrum", "saveTransitionCharges",
             "getTransitionDipolesExc")
    atomic = types.SimpleNamespace(valence_electrons={"h": 1, "c": 4}, atom_names=["h", "he", "li", "be", "b", "c"],
                                   ebohr_to_debye=2.541746)
    ns = {"np": np, "where": np.where, "argsort": np.argsort, "dot": np.dot, "meshgrid": np.meshgrid,
          "path": os.path, "AtomicData": atomic, "la": np.linalg}
    for n in names:
        exec(compile(method_source(lr, n, after=r"class LR_TDDFTB"), "LR_TDDFTB.py", "exec"), ns)
    Ref = type("LR_TDDFTB", (), {n: ns[n] for n in names})
    norb, nat = 14, 5
    orbe = np.sort(rng.standard_normal(norb))
    orbe[[2, 3]] = orbe[[3, 2]]  # occupations follow the energies, not the index order
    f = np.zeros(norb)
    f[np.argsort(orbe)[:6]] = 2.0
    orbs = np.linalg.qr(rng.standard_normal((norb, norb)))[0]
    X = rng.standard_normal((norb, norb, 3))
    D = X + X.transpose(1, 0, 2)
    pos = rng.standard_normal((nat, 3))
    atomlist = [(6, tuple(p)) for p in pos]
    dftb2 = types.SimpleNamespace(getOccupation=lambda: f, getKSEnergies=lambda: orbe,
                                  getDipoleMatrix=lambda: D, getKSCoefficients=lambda: orbs,
                                  getGeometry=lambda: atomlist, verbose=0, Nelec_val=12.0)
    r = Ref()
    r.dftb2 = dftb2
    r.setActiveOrbitals(nr_active_occ=3, nr_active_virt=4)
    C = rng.standard_normal((3, 3, 4))
    C /= np.sqrt((C * C).sum(axis=(1, 2)))[:, None, None]
    C[0] *= 0.0
    C[0, 2, 0], C[0, 1, 1] = np.sqrt(0.995), np.sqrt(0.005)
    r.Cij, r.Omega, r.multiplicity, r.Irreps = C, np.array([0.11, 0.17, 0.23]), "S", ["", "", ""]
    r.qtrans_ov = rng.standard_normal((nat, 3, 4))
    out = dict(orbe=orbe, f=f, orbs=orbs, D=D, pos=pos, C=C, Omega=r.Omega, qtrans_ov=r.qtrans_ov,
               occupied_orbs=r.occupied_orbs, virtual_orbs=r.virtual_orbs,
               active_occupied_orbs=r.active_occupied_orbs, active_virtual_orbs=r.active_virtual_orbs)
    r._TransitionDipolesMulliken()
    out["tdip_mulliken"] = np.array([r.tdipX, r.tdipY, r.tdipZ])
    r._TransitionDipoles()
    out["tdip"] = np.array([r.tdipX, r.tdipY, r.tdipZ])
    out["osc"] = r.getOscillatorStrengths()
    out["active_space_1e-5"] = np.array(r.determineActiveSpace())
    out["active_space_1e-2"] = np.array(r.determineActiveSpace(threshold=1e-2))
    import contextlib
    dftb2.verbose = 1
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        r.determineActiveSpace(threshold=1e-2)
    dftb2.verbose = 0
    out["active_space_text"] = np.array(buf.getvalue())
    out["tq_state_1"] = r.TransitionChargesState(1)
    # setActiveLMOrbitals on a planar-like C3H2 layout: the MO coefficients split into blocks over the p_z, the
    # s and the in-plane p atomic orbitals, so a selection of (l, m) keeps exactly the MOs of its blocks
    exec(compile(method_source(lr, "setActiveLMOrbitals", after=r"class LR_TDDFTB"), "LR_TDDFTB.py", "exec"), ns)
    sys.path.insert(0, REPO)
    from oracle import dftb_oracle as O
    valorbs = O.Parametrization([1, 6]).valorbs
    lm_atoms = [(6, (0.0, 0.0, 0.0)), (6, (2.6, 0.0, 0.0)), (6, (1.3, 2.2, 0.0)), (1, (-1.9, -0.5, 0.0)),
                (1, (4.5, -0.5, 0.0))]
    lms = [(l, m) for Z, _ in lm_atoms for (_, l, m) in valorbs[Z]]
    assert len(lms) == norb
    orbs_lm = np.zeros((norb, norb))
    cols = rng.permutation(norb)
    c0 = 0
    for block in ([(1, 0)], [(0, 0)], [(1, -1), (1, 1)]):
        rows = [k for k, lm in enumerate(lms) if lm in block]
        orbs_lm[np.ix_(rows, cols[c0:c0 + len(rows)])] = np.linalg.qr(rng.standard_normal((len(rows), len(rows))))[0]
        c0 += len(rows)
    assert c0 == norb
    lm_d = types.SimpleNamespace(getGeometry=lambda: lm_atoms, getValorbs=lambda: valorbs,
                                 getKSCoefficients=lambda: orbs_lm, getOccupation=lambda: f, getKSEnergies=lambda: orbe)
    import contextlib
    out.update(lm_orbs=orbs_lm, lm_Z=np.array([Z for Z, _ in lm_atoms]), lm_pos=np.array([p for _, p in lm_atoms]))
    for tag, sel in (("pz", [(1, 0)]), ("s_pz", [(0, 0), (1, 0)])):
        lm_r = types.SimpleNamespace(dftb2=lm_d)
        with contextlib.redirect_stdout(io.StringIO()):
            ns["setActiveLMOrbitals"](lm_r, nr_active_occ=2, nr_active_virt=3, select_lm=sel)
        out.update({"lm_%s_occupied" % tag: lm_r.occupied_orbs, "lm_%s_virtual" % tag: lm_r.virtual_orbs,
                    "lm_%s_active_occ" % tag: lm_r.active_occupied_orbs,
                    "lm_%s_active_virt" % tag: lm_r.active_virtual_orbs})
    out["tdip_exc"] = r.getTransitionDipolesExc(4)
    # the report printed at verbose > 0, with DFTBaby's AtomicData constants
    import contextlib
    ns["AtomicData"] = _reference_atomic_data(ref_root)
    dftb2.verbose = 1
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        r.getTransitionDipolesExc(4)
    dftb2.verbose = 0
    ns["AtomicData"] = atomic
    out["tdip_exc_report"] = np.array(buf.getvalue())
    tmp = tempfile.mkdtemp(prefix="dftbaby_lr_")
    real_string = sys.modules.get("string")
    sys.modules["string"] = types.SimpleNamespace(rjust=lambda text, width: text.rjust(width))
    try:
        r.saveAbsorptionSpectrum(os.path.join(tmp, "spec.dat"))
        r.saveTransitionCharges(os.path.join(tmp, "tq.dat"))
    finally:
        sys.modules["string"] = real_string
    out["spectrum_text"] = np.array(open(os.path.join(tmp, "spec.dat")).read())
    out["transition_charges_text"] = np.array(open(os.path.join(tmp, "tq.dat")).read())
    shutil.rmtree(tmp, ignore_errors=True)
    # the excitation table getEnergies prints at verbose > 0 (_dominant_excitations, _writeExcitations,
    # LR_TDDFTB.py:706-806), with utils.argsort_2d (utils.py:96-117; its integer division made explicit)
    for n in ("_dominant_excitations", "_writeExcitations"):
        exec(compile(method_source(lr, n, after=r"class LR_TDDFTB"), "LR_TDDFTB.py", "exec"), ns)
    ns_u = {"argsort": np.argsort}
    argsort_src = method_source(os.path.join(ref_root, "DFTB", "utils.py"), "argsort_2d")
    assert "sort_indx / ncols" in argsort_src
    exec(compile(argsort_src.replace("sort_indx / ncols", "sort_indx // ncols"), "utils.py", "exec"), ns_u)
    ad = _reference_atomic_data(ref_root)
    ns.update(utils=types.SimpleNamespace(argsort_2d=ns_u["argsort_2d"]), hartree_to_eV=ad.hartree_to_eV,
              hartree_to_nm=ad.hartree_to_nm)
    r._dominant_excitations = lambda I, dominant_probability=0.99: ns["_dominant_excitations"](r, I,
                                                                                               dominant_probability)
    dftb2.use_symmetry = 0
    r.Lambda2 = rng.random(3)
    r.en0 = -12.3456789
    r._TransitionDipoles()
    r.getOscillatorStrengths()
    out.update(Lambda2=r.Lambda2, en0=r.en0)
    for k, p in enumerate((0.99, 0.5)):
        for I in range(3):
            o, v, c = r._dominant_excitations(I, dominant_probability=p)
            out["domex_%d_%d" % (k, I)] = np.array([o, v, c], dtype=float)
    import contextlib
    sys.modules["string"] = types.SimpleNamespace(rjust=lambda text, width: text.rjust(width))
    try:
        for k, kw in enumerate((dict(), dict(nr_dominant_ex=3, print_MO_tdip=True),
                                dict(print_max_states=2, nr_dominant_ex=1))):
            buf = io.StringIO()
            with contextlib.redirect_stdout(buf):
                ns["_writeExcitations"](r, **kw)
            out["excitations_text_%d" % k] = np.array(buf.getvalue())
    finally:
        sys.modules["string"] = real_string
    np.savez_compressed(os.path.join(HERE, "lr_glue.npz"), **out)


def make_lambda(ref_root, rng):
    """DFTB2._construct_gaussian_overlap (DFTB2.py:1287-1317) on a C6H8 geometry with the Hubbard parameters
    of the shipped tables, and LR_TDDFTB._Lambda2_calcOia / _Lambda2_diagnostics (LR_TDDFTB.py:538-565) on
    synthetic diagonal transition charges with that overlap, run from DFTBaby's text."""
    sys.path.insert(0, REPO)
    from dftbaby_b200 import geometry
    from oracle import dftb_oracle as O
    ns = {"np": np, "zeros": np.zeros, "sqrt": np.sqrt, "log": np.log, "exp": np.exp, "dot": np.dot,
          "array": np.array, "pi": np.pi, "sum": np.sum}
    exec(compile(method_source(os.path.join(ref_root, "DFTB", "DFTB2.py"), "_construct_gaussian_overlap",
                               after=r"class DFTB2"), "DFTB2.py", "exec"), ns)
    for n in ("_Lambda2_calcOia", "_Lambda2_diagnostics"):
        exec(compile(method_source(os.path.join(ref_root, "DFTB", "LR_TDDFTB.py"), n, after=r"class LR_TDDFTB"),
                     "LR_TDDFTB.py", "exec"), ns)
    al = geometry.polyene(6, sigma=0.03, seed=21)
    par = O.Parametrization([1, 6])
    d = types.SimpleNamespace(atomlist=al, hubbard_U=par.hubbard_U)
    gaussOmega = ns["_construct_gaussian_overlap"](d)
    nat, no, nv, ns_ = len(al), 4, 5, 3
    q_oo = rng.standard_normal((nat, no, no))
    q_vv = rng.standard_normal((nat, nv, nv))
    C = rng.standard_normal((ns_, no, nv))
    td = types.SimpleNamespace(dftb2=types.SimpleNamespace(getGaussianOverlap=lambda: gaussOmega,
                                                           getGeometry=lambda: al),
                               active_occupied_orbs=np.arange(no), active_virtual_orbs=np.arange(no, no + nv),
                               qtrans_oo=q_oo, qtrans_vv=q_vv, Cij=C)
    ns["_Lambda2_calcOia"](td)
    Lambda2 = ns["_Lambda2_diagnostics"](td)
    np.savez_compressed(os.path.join(HERE, "lambda.npz"), Z=np.array([Z for Z, _ in al]),
                        pos=np.array([p for _, p in al]), gaussOmega=gaussOmega, q_oo=q_oo, q_vv=q_vv, C=C,
                        Oia=td.Oia, Lambda2=Lambda2)


def _reference_atomic_data(ref_root):
    """DFTB/AtomicData.py executed through the shim (names, masses, conversion factors)."""
    ns = {}
    exec(compile(py2to3(open(os.path.join(ref_root, "DFTB", "AtomicData.py")).read()), "AtomicData.py", "exec"), ns)
    return types.SimpleNamespace(**{k: v for k, v in ns.items() if not k.startswith("__")})


def make_particle_hole(ref_root, rng):
    """LR_TDDFTB.ParticleHoleCharges, ParticleHoleChargesSuperposition and analyseParticleHole
    (LR_TDDFTB.py:910-1007) run from DFTBaby's text on the C4H6 layout of make_mulliken_trans_charges,
    with the Mulliken transition charges q_oo, q_vv made by DFTBaby's own Python loop
    (LR_TDDFTB.py:267-296) from the stored S and orbitals."""
    import textwrap
    Zs = [6, 6, 6, 6, 1, 1, 1, 1, 1, 1]
    valorbs = {1: [(1, 0, 0)], 6: [(2, 0, 0), (2, 1, -1), (2, 1, 0), (2, 1, 1)]}
    pos = rng.standard_normal((len(Zs), 3)) * 2.0
    atomlist = [(Z, tuple(p)) for Z, p in zip(Zs, pos)]
    norb = sum(len(valorbs[Z]) for Z in Zs)
    X = rng.standard_normal((norb, norb))
    S = np.eye(norb) + 0.05 * (X + X.T)
    orbs = np.linalg.qr(rng.standard_normal((norb, norb)))[0]
    occ, virt = np.array([2, 4, 5, 7, 8]), np.array([11, 12, 15, 19])
    lines = open(os.path.join(ref_root, "DFTB", "LR_TDDFTB.py")).read().expandtabs(8).splitlines(keepends=True)
    start = next(i for i, ln in enumerate(lines) if ln.strip() == "# PYTHON CODE")
    end = next(i for i in range(start + 1, len(lines)) if lines[i].strip() == '"""')
    block = py2to3(textwrap.dedent("".join(lines[start:end])))
    nst = 3
    C = rng.standard_normal((nst, len(occ), len(virt)))
    C /= np.sqrt((C * C).sum(axis=(1, 2)))[:, None, None]
    coeffs = rng.standard_normal(nst) + 1j * rng.standard_normal(nst)
    r = types.SimpleNamespace(active_occupied_orbs=occ, active_virtual_orbs=virt, Cij=C, Omega=np.array([0.1, 0.2, 0.3]),
                              dftb2=types.SimpleNamespace(getGeometry=lambda: atomlist, verbose=0))
    ns = {"zeros": np.zeros, "dot": np.dot, "self": r, "atomlist": atomlist, "valorbs": valorbs, "orbs": orbs,
          "S": S}
    exec(compile(block, "LR_TDDFTB.py:_MullikenTransitionCharges", "exec"), ns)
    ns = {"np": np, "la": np.linalg, "path": os.path, "atom_names": ["h", "he", "li", "be", "b", "c"],
          "string": types.SimpleNamespace(center=lambda text, width: text.center(width))}
    for n in ("ParticleHoleCharges", "ParticleHoleChargesSuperposition", "analyseParticleHole"):
        exec(compile(method_source(os.path.join(ref_root, "DFTB", "LR_TDDFTB.py"), n, after=r"class LR_TDDFTB"),
                     "LR_TDDFTB.py", "exec"), ns)
    r.ParticleHoleCharges = lambda I: ns["ParticleHoleCharges"](r, I)
    ph = [ns["ParticleHoleCharges"](r, I) for I in range(nst)]
    sup_p, sup_h = ns["ParticleHoleChargesSuperposition"](r, coeffs)
    tmp = tempfile.mkdtemp(prefix="dftbaby_ph_")
    ns["analyseParticleHole"](r, particle_hole_states=[1, 3], particle_hole_dir=tmp)
    chrg = [open(os.path.join(tmp, "particle_hole_charges_%d.chrg" % I)).read() for I in (1, 3)]
    # the exciton reports printed at verbose > 0
    import contextlib
    r.dftb2.verbose = 1
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        ns["ParticleHoleCharges"](r, 1)
        ns["ParticleHoleChargesSuperposition"](r, coeffs)
    r.dftb2.verbose = 0
    report = buf.getvalue()
    shutil.rmtree(tmp, ignore_errors=True)
    np.savez_compressed(os.path.join(HERE, "particle_hole.npz"), Z=np.array(Zs), pos=pos, S=S, orbs=orbs, occ=occ,
                        virt=virt, C=C, coeffs=coeffs, ph_p=np.array([p for p, _ in ph]),
                        ph_h=np.array([h for _, h in ph]), sup_p=sup_p, sup_h=sup_h, chrg_1=np.array(chrg[0]),
                        chrg_3=np.array(chrg[1]), report=np.array(report))


def make_dftb2_props(ref_root, rng):
    """DFTB2.getDipoleMoment, getMullikenDipoleMoment (with _center_of_nuclear_charge), write_Mulliken_charges,
    _balance_partial_charges and setCharge (DFTB2.py:429-435, 839-860, 1712-1721, 2456-2486) run from DFTBaby's
    text on a stand-in C2H4 ground state: random symmetric density and dipole matrices, Mulliken populations."""
    import contextlib
    names = ("getDipoleMoment", "getMullikenDipoleMoment", "_center_of_nuclear_charge", "write_Mulliken_charges",
             "_balance_partial_charges", "setCharge")
    ns = {"np": np, "zeros": np.zeros, "array": np.array, "sum": np.sum,
          "atom_names": ["h", "he", "li", "be", "b", "c"]}
    for n in names:
        exec(compile(method_source(os.path.join(ref_root, "DFTB", "DFTB2.py"), n, after=r"class DFTB2"), "DFTB2.py",
                     "exec"), ns)
    Ref = type("DFTB2", (), {n: ns[n] for n in names})
    Zs = [6, 6, 1, 1, 1, 1]
    pos = rng.standard_normal((len(Zs), 3)) * 1.5
    norb = 12
    X = rng.standard_normal((norb, norb))
    P = X + X.T
    X = rng.standard_normal((norb, norb, 3))
    D = X + X.transpose(1, 0, 2)
    q0 = np.array([4.0, 4.0, 1.0, 1.0, 1.0, 1.0])
    dq = 0.1 * rng.standard_normal(len(Zs))
    r = Ref()
    r.atomlist = [(Z, tuple(p)) for Z, p in zip(Zs, pos)]
    r.P, r.q0, r.dq, r.q = P, q0, dq, q0 - dq
    r.getDipoleMatrix = lambda: D
    out = dict(Z=np.array(Zs), pos=pos, P=P, D=D, q0=q0, dq=dq)
    with contextlib.redirect_stdout(io.StringIO()):
        out["dipole"] = r.getDipoleMoment()  # the reference also prints P here
    r._center_of_nuclear_charge()
    out["Rcc"], out["mulliken_dipole"] = r.Rcc, r.getMullikenDipoleMoment()
    real_string = sys.modules.get("string")
    sys.modules["string"] = types.SimpleNamespace(center=lambda text, width: text.center(width))
    buf = io.StringIO()
    try:
        with contextlib.redirect_stdout(buf):
            r.write_Mulliken_charges()
    finally:
        sys.modules["string"] = real_string
    out["mulliken_text"] = np.array(buf.getvalue())
    for k, charge in enumerate((0.0, 1.0, -2.0)):
        r.charge = charge
        r.dq = dq.copy()
        r._balance_partial_charges()
        out["balanced_%d" % k] = r.dq
        buf = io.StringIO()
        with contextlib.redirect_stdout(buf):
            r.setCharge(charge)
        out["nelec_%d" % k], out["setcharge_text_%d" % k] = r.Nelec_val, np.array(buf.getvalue())
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        r.setCharge(12.0)  # no valence electrons left: the reference warns
    out["nelec_empty"], out["setcharge_text_empty"] = r.Nelec_val, np.array(buf.getvalue())
    # the report of one SCC iteration printed at verbose > 0 (DFTB2.writeIteration, DFTB2.py:2146-2233)
    exec(compile(method_source(os.path.join(ref_root, "DFTB", "DFTB2.py"), "writeIteration", after=r"class DFTB2"),
                 "DFTB2.py", "exec"), ns)
    ns.update(hartree_to_eV=_reference_atomic_data(ref_root).hartree_to_eV, argsort=np.argsort)
    orbe = np.sort(rng.standard_normal(12))[rng.permutation(12)]
    it = types.SimpleNamespace(i=7, relative_change=3.25e-6, E_bs=-11.1, E_coulomb=0.05, E_HF_x=-0.02,
                               E_elec=-11.07, E_rep=0.8, E_tot=-10.27, HLgap=0.31, orbe=orbe,
                               f=np.where(orbe < np.sort(orbe)[6], 2.0, 0.0), q=q0 - dq, dq=dq, verbose=1,
                               mulliken_dipoles=0, qmmm=None, cavity=None, atomlist=r.atomlist)
    sys.modules["string"] = types.SimpleNamespace(center=lambda text, width: text.center(width),
                                                  rjust=lambda text, width: text.rjust(width))
    buf = io.StringIO()
    try:
        with contextlib.redirect_stdout(buf):
            ns["writeIteration"](it)
    finally:
        sys.modules["string"] = real_string
    out.update(it_orbe=orbe, it_f=it.f, iteration_text=np.array(buf.getvalue()))
    np.savez_compressed(os.path.join(HERE, "dftb2_props.npz"), **out)


XYZ_TEXT = """6
charge=+1 name=ethene tags=[1,2] note=C2H4
C      0.000000    0.000000    0.667480
C      0.000000    0.000000   -0.667480
H      0.000000    0.922832    1.237695
H      0.000000   -0.922832    1.237695
H1     0.000000    0.922832   -1.237695
h      0.000000   -0.922832   -1.237695
Tv     2.5  0.0  0.0
6
second frame
C      0.010000    0.000000    0.667480
C      0.000000    0.020000   -0.667480
H      0.000000    0.922832    1.237695
H      0.000000   -0.922832    1.237695
H      0.000000    0.922832   -1.237695
H      0.000000   -0.922832   -1.237695
"""


def make_repulsive(ref_root, rng):
    """RepulsivePotential.__init__ / getVrep (RepulsivePotential.py:17-100, as DFTB2.py:327 builds them: no
    smooth tail) on the shipped H-H, H-C and C-C tables, run from DFTBaby's text: values and first
    derivatives below the grid, inside it and beyond its last point."""
    from collections import defaultdict
    from scipy import interpolate
    rp = os.path.join(ref_root, "DFTB", "RepulsivePotential", "RepulsivePotential.py")
    ns = {"np": np, "interpolate": interpolate, "defaultdict": defaultdict, "argmax": np.argmax,
          "exp": np.exp, "pow": pow}
    for n in ("__init__", "getVrep"):
        exec(compile(method_source(rp, n, after=r"class RepulsivePotential"), "RepulsivePotential.py", "exec"), ns)
    RP = type("RepulsivePotential", (), {"__init__": ns["__init__"], "getVrep": ns["getVrep"]})
    out = {}
    for name in ("h_h", "h_c", "c_c"):
        path = os.path.join(ref_root, "DFTB", "RepulsivePotential", "reppot_tables", name + ".py")
        mod = types.ModuleType(name)
        exec(compile(open(path).read(), path, "exec"), mod.__dict__)
        pot = RP(mod)
        R = np.sort(np.concatenate([rng.uniform(0.6 * pot.dmin, pot.dmin, 3), rng.uniform(pot.dmin, pot.dmax, 25),
                                    [pot.dmax, pot.dmax * 1.2]]))
        import contextlib
        with contextlib.redirect_stdout(io.StringIO()):  # the reference warns below the grid
            out[name + "_R"] = R
            out[name + "_V"] = np.array([float(pot.getVrep(r)) for r in R])
            out[name + "_dV"] = np.array([float(pot.getVrep(r, deriv=1)) for r in R])
        out[name + "_Z"] = np.array([mod.Z1, mod.Z2])
    np.savez_compressed(os.path.join(HERE, "repulsive.npz"), **out)


def make_lr_e2e(ref_root, mods):
    """LR_TDDFTB.getEnergies end to end from DFTBaby's text (LR_TDDFTB.py:167-188, 254-320, 378-527, 538-705,
    741-758 and determineActiveSpace) over the reference SCC stand-in (``_reference_dftb2``) and the shimmed
    Solver module, on the oracle's S, H0, D, gamma, gamma_lr and Gaussian overlap.  The Fortran
    tddftb.trans_charges is served by the oracle's restatement (pinned against the reference's Python twin);
    getTransitionDipolesExc (excited-excited dipoles, not used for Omega and f) is skipped.  Cases: C6H8
    without long-range correction (Hermitian Davidson), C6H8 with it (non-Hermitian Davidson) and C4H6 with
    it solved by full Casida."""
    import importlib

    from dftbaby_b200 import geometry
    from oracle import dftb_oracle as O
    ext = importlib.import_module("DFTB.extensions")
    ext.tddftb = types.SimpleNamespace(tddftb=types.SimpleNamespace(
        trans_charges=lambda oo, ov, S, opa: O.trans_charges(np.ascontiguousarray(oo), np.ascontiguousarray(ov),
                                                             np.ascontiguousarray(S), np.asarray(opa, np.int32))))
    Ref = _reference_dftb2(ref_root, mods)
    lr = os.path.join(ref_root, "DFTB", "LR_TDDFTB.py")
    names = ("setActiveOrbitals", "setMultiplicity", "_solve_lr_equations", "_MullikenTransitionCharges",
             "_Lambda2_calcOia", "_Lambda2_diagnostics", "_getOrbitalEnDifferences", "_getOrbitalOccDifferences",
             "_TransitionDipoles", "getOscillatorStrengths", "_SymmetryOfExcitations", "determineActiveSpace",
             "getEnergies")
    ns = {"np": np, "la": np.linalg, "array": np.array, "where": np.where, "argsort": np.argsort,
          "zeros": np.zeros, "dot": np.dot, "tensordot": np.tensordot, "transpose": np.transpose,
          "diag": np.diag, "reshape": np.reshape, "sqrt": np.sqrt, "arange": np.arange, "outer": np.outer,
          "sum": np.sum, "meshgrid": np.meshgrid, "eigh": np.linalg.eigh, "path": os.path,
          "Solver": mods["Solver"], "StabilityAnalysis": None, "LongRangeCTCorrection": None,
          "SymmetryAssignmentEx": None}
    for n in names:
        exec(compile(method_source(lr, n, after=r"class LR_TDDFTB"), "LR_TDDFTB.py", "exec"), ns)
    LR = type("LR_TDDFTB", (), dict({n: ns[n] for n in names}, getTransitionDipolesExc=lambda self, Nst: None))
    out = {}
    cases = (("c6h8", geometry.polyene(6, sigma=0.02, seed=31), 0, 4),
             ("c6h8_lc", geometry.polyene(6, sigma=0.02, seed=32), 1, 4),
             ("c4h6_lc_casida", geometry.polyene(4, sigma=0.02, seed=33), 1, None))
    for name, al, lc, nstates in cases:
        od = O.DFTB2(al, long_range_correction=lc)
        od.setGeometry(al)
        od.getEnergy()
        d = Ref()
        _load_into(d, od, lc)
        d.D, d.gaussOmega, d.parameter_set, d.use_symmetry = od.D, od.gaussOmega, "homegrown", 0
        d.getEnergy = types.MethodType(lambda self, **opts: (self.runSCC(**opts), 0.0)[1], d)
        for acc, attr in (("getKSEnergies", "orbe"), ("getOccupation", "f"), ("getKSCoefficients", "orbs"),
                          ("getGeometry", "atomlist"), ("getValorbs", "valorbs"), ("getOverlapMatrix", "S"),
                          ("getGamma", "gamma"), ("getGamma_lr", "gamma_lr"), ("getDipoleMatrix", "D"),
                          ("getGaussianOverlap", "gaussOmega")):
            setattr(d, acc, (lambda a: (lambda: getattr(d, a)))(attr))
        td = LR()
        td.dftb2, td.XmY, td.XpY, td.Omega = d, None, None, None
        opts = dict(nstates=nstates, diag_conv=1.0e-10, diag_maxiter=100)
        Om, f = td.getEnergies(**opts)
        out["%s_Z" % name] = np.array([Z for Z, _ in al])
        out["%s_pos" % name] = np.array([p for _, p in al])
        out["%s_lc" % name] = lc
        out["%s_nstates" % name] = -1 if nstates is None else nstates
        out["%s_Omega" % name], out["%s_f" % name] = np.asarray(Om), np.asarray(f)
        out["%s_Lambda2" % name] = np.asarray(td.Lambda2)
        n = len(Om) if nstates is None else nstates
        out["%s_tdip" % name] = np.array([td.tdipX[:n], td.tdipY[:n], td.tdipZ[:n]])
    np.savez_compressed(os.path.join(HERE, "lr_e2e.npz"), **out)


PARTS = ("sk_rules", "gamma", "diis", "solvers", "sk_grad_rules", "gradients")


def main(ref_root, only=None):
    sys.path.insert(0, REPO)
    rng = np.random.default_rng(20261203)
    tmp, mods = load_reference_modules(ref_root)
    try:
        if only in (None, "core"):
            make_sk_rules(ref_root, rng)
            make_gamma(mods, rng)
            make_diis(mods, rng)
            make_solvers(mods, rng)
            make_sk_grad_rules(ref_root, rng)
            make_gradients(mods, rng)
        if only in (None, "couplings"):
            make_couplings(ref_root, np.random.default_rng(20261204))
        if only in (None, "mulliken"):
            make_mulliken_trans_charges(ref_root, np.random.default_rng(20261205))
        if only in (None, "sk_python"):
            make_sk_python(ref_root, np.random.default_rng(20261206))
        if only in (None, "scc"):
            make_scc(ref_root, mods)
        if only in (None, "lr_glue"):
            make_lr_glue(ref_root, np.random.default_rng(20261207))
        if only in (None, "lambda"):
            make_lambda(ref_root, np.random.default_rng(20261208))
        if only in (None, "repulsive"):
            make_repulsive(ref_root, np.random.default_rng(20261209))
        if only in (None, "lr_e2e"):
            make_lr_e2e(ref_root, mods)
        if only in (None, "particle_hole"):
            make_particle_hole(ref_root, np.random.default_rng(20261210))
        if only in (None, "dftb2_props"):
            make_dftb2_props(ref_root, np.random.default_rng(20261212))
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--only=")]
    only = next((a.split("=", 1)[1] for a in sys.argv[1:] if a.startswith("--only=")), None)
    if len(args) != 1:
        sys.exit("usage: python make_golden.py REFERENCE_ROOT [--only=PART]  (REFERENCE_ROOT: the DFTBaby checkout)")
    main(args[0], only)
