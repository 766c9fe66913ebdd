"""The C-ABI library loads without a GPU and exports every entry point the
public headers declare (no compute calls)."""

import ctypes as ct
import glob
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\**\s+\**(az_[A-Za-z0-9_]+)\s*\(",
                             src, flags=re.M):
            names.add(m.group(1))
    return names


def test_header_declares_entry_points():
    names = declared_functions()
    assert "az_euler_dudt" in names and "az_rk3_integrate" in names and "az_fft_forward" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    lib = ct.CDLL(os.path.join(ROOT, "azeban_b200", "libazeban_b200.so"))
    missing = [n for n in sorted(declared_functions()) if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_lists_every_symbol():
    from azeban_b200 import _lib
    assert set(_lib.EXPORTS) == declared_functions()


def test_supported_lengths_without_gpu():
    import azeban_b200 as az
    lens = az.supported_lengths()
    for M in (96, 192, 384, 768):
        assert M in lens


def test_host_side_config_mirrors_reference():
    import azeban_b200 as az
    g = az.make_grid({"N_phys": 256, "N_phys_pad": ""}, 3)
    assert (g.N_phys, g.N_phys_pad, g.N_fourier, g.N_fourier_pad) == (256, 384, 129, 193)
    g2 = az.make_grid({"N_fourier": 33}, 2)
    assert (g2.N_phys, g2.N_phys_pad) == (64, 96)
    v = az.make_viscosity({"type": "Smooth Cutoff", "eps": 0.05}, g)
    assert abs(v.eps - 0.05 / 256) < 1e-18 and abs(v.k0 - 2 * 3.141592653589793 * 16) < 1e-12
    q = az.make_viscosity({"type": "Quadratic", "eps": 0.05}, g)
    assert q.N == 256 and abs(q.eps - 0.05 / 256) < 1e-18
    import pytest
    with pytest.raises(ValueError):
        az.make_viscosity({"type": "Smooth Cutoff"}, g)
    with pytest.raises(ValueError):
        az.make_grid({"N_phys": 8, "N_fourier": 5}, 2)


def test_philox_known_answers():
    """The random stream's block function, Philox4x32-10, against the
    known-answer vectors its authors publish with the algorithm (counter,
    key -> output); a host call, no GPU."""
    import ctypes as ct
    from azeban_b200 import _lib
    kat = [
        ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
        ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
        ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
         (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
    ]
    for ctr, key, want in kat:
        out = (ct.c_uint * 4)()
        _lib.check(_lib.lib.az_philox4x32_10((ct.c_uint * 4)(*ctr), (ct.c_uint * 2)(*key), out))
        assert tuple(out) == want
