"""CPU tests of the product library: it loads without a GPU, exports every
entry point of include/eup.h, reads and writes the reference's file formats,
and builds the synthetic inputs bit-identically to the oracle."""
import ctypes
import os
import re
import struct

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    txt = open(os.path.join(ROOT, "include", "eup.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(eup_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_header_symbol(eup):
    names = header_functions()
    assert len(names) >= 25
    lib = ctypes.CDLL(eup.LIB_PATH)
    for nm in names:
        assert hasattr(lib, nm), nm
    assert sorted(eup.EXPORTED) == names


def test_abi_version_and_no_device_paths(eup):
    assert eup.lib.eup_abi_version() == 1
    if eup.device_count() == 0:
        with pytest.raises(eup.EupError) as e:
            eup.Solver(eup.Config(8, 8, 8))
        assert e.value.code == 7


def test_create_rejects_bad_flags(eup):
    for bc in ((4, 4, 3, 3, 0, 0), (5, 5, 3, 3, 0, 0), (5, 4, 2, 3, 0, 0), (5, 4, 3, 3, 0, 4)):
        with pytest.raises(eup.EupError) as e:
            eup.Solver(eup.Config(8, 8, 8, bc=bc))
        assert e.value.code == 5


def test_init_matches_oracle_bit_exact(eup, orc):
    for dt in (np.float32, np.float64):
        a = eup.init_equilibrium(11, 7, 5, 0.05, 1e-4, 1234, dt)
        b = orc.init_perturbed(11, 7, 5, 0.05, 1e-4, 1234, dt)
        assert np.array_equal(a, b)


def test_raw_state_round_trip_and_layout(eup, tmp_path):
    a = eup.init_equilibrium(6, 5, 4, 0.05, 1e-3, 3)
    p = tmp_path / "save.00.00.00.00000042.bin"
    eup.write_raw_state(p, a, 42)
    raw = p.read_bytes()
    # record 1: itime (CODE/SRC/save_raw.F90:54), then 19 records of (l+2)(m+2)(n+2) reals
    assert struct.unpack("<iii", raw[:12]) == (4, 42, 4)
    rec = 8 * 7 * 6 * 4
    assert struct.unpack("<i", raw[12:16])[0] == rec
    assert len(raw) == 12 + 19 * (rec + 8)
    first = np.frombuffer(raw[16:16 + rec], dtype=np.float32)
    assert np.array_equal(first, a[0].ravel())
    b, it = eup.read_raw_state(p, 6, 5, 4)
    assert it == 42 and np.array_equal(a, b)
    with pytest.raises(eup.EupError) as e:
        eup.read_raw_state(p, 6, 5, 5)
    assert e.value.code == 6


def test_obs_file_round_trip(eup, tmp_path):
    obs = np.zeros((4, 5, 6), np.int32)
    obs[1, 2, 3] = obs[3, 4, 5] = obs[0, 0, 0] = 1
    p = tmp_path / "obs.0000.00000000.bin"
    eup.write_obs_file(p, obs)
    raw = p.read_bytes()
    assert struct.unpack("<iii", raw[:12]) == (4, 3, 4)
    # entries in k, j, i order with 1-based indices (CODE/SRC/build.obs.F90:523-530)
    assert struct.unpack("<iiiii", raw[12:32]) == (12, 1, 1, 1, 12)
    back, cnt = eup.read_obs_file(p, 6, 5, 4)
    assert cnt == 3 and np.array_equal(back, obs)
    p.write_bytes(raw[:-3])
    with pytest.raises(eup.EupError):
        eup.read_obs_file(p, 6, 5, 4)


def test_geometry_cylinder(eup):
    obs = eup.geometry_cylinder_z(40, 30, 3, 20, 15, 5)
    k, j, i = np.meshgrid(np.arange(1, 4), np.arange(1, 31), np.arange(1, 41), indexing="ij")
    assert np.array_equal(obs, ((i - 20) ** 2 + (j - 15) ** 2 <= 25).astype(np.int32))


def test_geometry_reticular_shell(eup):
    l, m, n = 160, 72, 72
    obs = eup.geometry_reticular_shell(l, m, n, 40, 64, 36.5, 36.5, 48, 4, 16, 7)
    assert obs.any()
    k, j, i = np.nonzero(obs)
    r = np.sqrt((j + 1 - 36.5) ** 2 + (k + 1 - 36.5) ** 2)
    assert r.max() <= 24 + 1e-9 and r.min() >= 20 - 1e-9   # within the strut annulus
    assert (i + 1).min() >= 38 and (i + 1).max() <= 40 + 64 + 2
    # the seed moves the grid, the same seed reproduces it
    assert np.array_equal(obs, eup.geometry_reticular_shell(l, m, n, 40, 64, 36.5, 36.5, 48, 4, 16, 7))
    assert not np.array_equal(obs, eup.geometry_reticular_shell(l, m, n, 40, 64, 36.5, 36.5, 48, 4, 16, 8))
    # a lattice shell, not a tube: a good part of the annulus stays open
    jj, kk = np.meshgrid(np.arange(1, m + 1), np.arange(1, n + 1))
    rr = np.sqrt((jj - 36.5) ** 2 + (kk - 36.5) ** 2)
    ann = ((rr >= 20.5) & (rr <= 23.5)).sum() * 64
    assert 0.2 < obs[:, :, 40:104].sum() / ann < 0.9


def test_geometry_ridged_shell(eup):
    l, m, n = 160, 72, 72
    args = (l, m, n, 40, 64, 36.5, 36.5, 48, 4, 16)
    shell = eup.geometry_reticular_shell(*args, 7)
    hard = eup.geometry_ridged_shell(*args, 4.0, 3.0, 4.0, 5.0, 0.0, 7)
    assert set(np.unique(hard)) <= {0.0, 1.0}
    # the shell is kept; ridges and cap only add solid
    assert np.all(hard[shell == 1] == 1.0)
    extra = (hard == 1.0) & (shell == 0)
    k, j, i = np.nonzero(extra)
    r = np.sqrt((j + 1 - 36.5) ** 2 + (k + 1 - 36.5) ** 2)
    ridge = r >= 23.5                                            # ridges start half a voxel inside Ro
    assert ridge.any() and r[ridge].max() <= 24 + 4 + 1e-9      # and stand at most ridge_h proud
    cap = ~ridge
    assert cap.any() and (i[cap] + 1).min() >= 40 + 64 - 4 - 1   # the cap closes the last cap_t of the body
    # the porous cap has open pores
    capsl = hard[:, :, 104 - 3:104]
    jj, kk = np.meshgrid(np.arange(1, m + 1), np.arange(1, n + 1))
    inside = np.sqrt((jj - 36.5) ** 2 + (kk - 36.5) ** 2) < 20
    assert 0.1 < 1.0 - capsl[inside].mean() < 0.9
    # smooth field: d ns / d h matches a central difference
    ns, d = eup.geometry_ridged_shell(*args, 4.0, 3.0, 4.0, 5.0, 1.0, 7, with_derivative=True)
    assert ns.min() >= 0.0 and ns.max() <= 1.0 and (d > 0).any()
    hp = eup.geometry_ridged_shell(*args, 4.0 + 1e-5, 3.0, 4.0, 5.0, 1.0, 7)
    hm = eup.geometry_ridged_shell(*args, 4.0 - 1e-5, 3.0, 4.0, 5.0, 1.0, 7)
    fd = (hp - hm) / 2e-5
    assert np.abs(fd - d).max() < 1e-5 * max(1.0, np.abs(d).max())


def _c_prototypes():
    """name -> list of parameter declarations of every function in include/eup.h."""
    src = open(os.path.join(ROOT, "include", "eup.h")).read()
    src = re.sub(r"/\*.*?\*/", " ", src, flags=re.S)
    src = re.sub(r"\s+", " ", src)
    out = {}
    for ret, name, params in re.findall(r"(int|int32_t|const char ?\*|uint64_t) ?(eup_[a-z0-9_]+)\(([^)]*)\);", src):
        ps = [x.strip() for x in params.split(",")] if params.strip() not in ("", "void") else []
        out[name] = ps
    return out


def _fortran_interfaces():
    """name -> list of (dummy name, declaration line) of every bind(c) function in eup_mod.F90."""
    src = open(os.path.join(ROOT, "fortran", "eup_mod.F90")).read()
    out = {}
    for m in re.finditer(r'function (eup_[a-z0-9_]+)\(([^)]*)\)\s*&?\s*bind\(c,\s*name="(eup_[a-z0-9_]+)"\)(.*?)end function',
                         src, flags=re.S):
        dummies = [d.strip() for d in m.group(2).replace("&", " ").split(",") if d.strip()]
        decls = {}
        for line in m.group(4).splitlines():
            line = line.split("!")[0]
            if "::" not in line:
                continue
            spec, names = line.split("::", 1)
            for nm in re.findall(r"([a-z_0-9]+)\s*(?:\([^)]*\))?", names):
                decls[nm] = spec.strip()
        out[m.group(3)] = [(d, decls.get(d, "")) for d in dummies]
    return out


def test_fortran_interfaces_match_the_c_prototypes():
    """Argument by argument (there is no Fortran compiler here to check the module): the same
    count; a C scalar passed by value (int32_t, int64_t, uint64_t, double) is declared `value`
    with the matching interop kind; a C pointer is not passed by value unless it is declared
    type(c_ptr)."""
    c, f = _c_prototypes(), _fortran_interfaces()
    assert sorted(c) == sorted(f) == header_functions()
    kinds = {"int32_t": "c_int32_t", "int64_t": "c_int64_t", "uint64_t": "c_int64_t", "double": "c_double"}
    for name, params in c.items():
        dummies = f[name]
        assert len(params) == len(dummies), (name, params, dummies)
        for p, (dn, decl) in zip(params, dummies):
            assert decl, (name, dn, "undeclared dummy")
            pointer = "*" in p or "[" in p
            if pointer:
                assert ("value" not in decl) or ("c_ptr" in decl) or ("c_funptr" in decl), (name, p, decl)
            else:
                ctype = p.split()[-2] if len(p.split()) > 1 else p
                assert "value" in decl, (name, p, decl)
                assert kinds[ctype] in decl, (name, p, decl)


def test_fortran_module_binds_every_entry_point():
    """fortran/eup_mod.F90 declares a bind(c) interface, once, for every function of include/eup.h
    (it is not compiled here: there is no Fortran compiler), in free-form lines of at most 132
    characters."""
    src = open(os.path.join(ROOT, "fortran", "eup_mod.F90")).read()
    bound = re.findall(r'bind\(c,\s*name="(eup_[a-z0-9_]+)"\)', src)
    assert sorted(bound) == header_functions()
    assert max(len(line) for line in src.splitlines()) <= 132
