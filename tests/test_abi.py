"""CPU checks of the drop-in boundary: the sm_100a library loads and exports every symbol that
include/safire_b200.h declares, and the Python binding covers them.  No compute call is made."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "safire_b200.h")


def declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|size_t|const char\*|void\*)\s+(sfq_\w+)\s*\(", text, re.M)))


@pytest.fixture(scope="module")
def lib():
    from safire_b200 import build
    path = build.build()
    return ctypes.CDLL(path)


def test_header_declares_entry_points():
    names = declared()
    assert len(names) >= 25
    for n in ("sfq_mixed_density_matrix", "sfq_log_overlap", "sfq_propagate", "sfq_orthogonalize", "sfq_vbias",
              "sfq_vhs", "sfq_energy", "sfq_assemble_x", "sfq_comb", "sfq_engine_create", "sfq_engine_propagate",
              "sfq_engine_run"):
        assert n in names


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    from safire_b200 import capi
    assert set(declared()) <= set(capi.exported_symbols())


def test_last_error_and_version(lib):
    from safire_b200 import capi
    L = capi.lib()
    assert L.sfq_abi_version() == 13
    assert isinstance(L.sfq_last_error(), bytes)


def test_argument_errors_without_gpu():
    """Shape / null checks return codes before any device work."""
    from safire_b200 import capi
    L = capi.lib()
    assert L.sfq_mixed_density_matrix(None, 0, None, None, None, -1, 4, 2, 1, None, 0, None) == 1
    assert L.sfq_mixed_density_matrix(None, 0, None, None, None, 3, 4, 2, 1, None, 0, None) == 2
    assert L.sfq_vbias(None, None, 0, None, 2, 2, 4, 0, 0.01, 1, None) == 0  # empty: no-op
    p = capi.default_params(nmo=4, nel=8, nchol=3, nwalk=2)
    h = ctypes.c_void_p()
    import numpy as np
    z = np.zeros(64)
    rc = L.sfq_engine_create(ctypes.byref(h), ctypes.byref(p), z.ctypes.data, z.ctypes.data, z.ctypes.data)
    assert rc == 1  # nel > nmo: SFQ_ERR_SHAPE


def test_workspace_sizes_monotone():
    from safire_b200 import capi
    L = capi.lib()
    a = L.sfq_workspace_size(capi.OP_MIXED_DENSITY_MATRIX, 8, 40, 10, 0)
    b = L.sfq_workspace_size(capi.OP_MIXED_DENSITY_MATRIX, 16, 40, 10, 0)
    assert 0 < a < b
    assert L.sfq_workspace_size(capi.OP_ENERGY, 8, 40, 10, 100) > 0


def test_group_and_tiles_argument_errors_without_gpu():
    from safire_b200 import capi
    L = capi.lib()
    g = ctypes.c_void_p()
    assert L.sfq_group_create(ctypes.byref(g), None, 0) == 2
    arr = (ctypes.c_void_p * 2)(None, None)
    assert L.sfq_group_create(ctypes.byref(g), arr, 2) == 2
    assert L.sfq_group_destroy(None) == 0
    assert L.sfq_group_block_query(None) == 2
    assert L.sfq_engine_autotune(None, 3, None) == 2
    assert L.sfq_engine_set_tiles(None, None) == 2


def test_uneven_systems_layout():
    """24 systems: M = 48..320 in steps of 16, cycled; N = M/4; Nchol = 5M; walkers in [64, 512]."""
    from safire_b200 import batched
    specs, walkers = batched.uneven_specs(24)
    assert [s.M for s in specs] == [48 + 16 * (i % 18) for i in range(24)]
    assert all(s.N * 4 == s.M and s.Nc == 5 * s.M for s in specs)
    assert all(64 <= w <= 512 for w in walkers) and len(set(walkers)) > 12


def test_cpp_header_compiles():
    """include/safire_b200.hpp (the reference-named C++ view) is valid C++17 against the C header."""
    import shutil
    import subprocess
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no g++")
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
    src = '#include "safire_b200.hpp"\nint main() { return 0; }\n'
    r = subprocess.run([gxx, "-std=c++17", "-fsyntax-only", "-I", inc, "-x", "c++", "-"], input=src,
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_cpp_population_planning_runs_on_the_host(tmp_path):
    """A C++ program using the reference-named comb and plan_walker_exchange of safire_b200.hpp,
    linked against the library, runs on the CPU (host-only entry points) and agrees with the oracle."""
    import shutil
    import subprocess
    import numpy as np
    from oracle import afqmc_oracle as O
    from safire_b200 import build
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no g++")
    lib = build.build()
    src = r'''
#include <cstdio>
#include "safire_b200.hpp"
int main() {
  std::vector<double> w;
  for (int i = 0; i < 24; ++i) w.push_back((i % 5 == 0) ? 0.0 : 0.25 * ((i * 7) % 11 + 1));
  std::vector<int> off = safire_b200::comb(w, 0.3125, 24);
  for (int k : off) std::printf("%d ", k);
  std::printf("\n");
  for (auto t : safire_b200::plan_walker_exchange(off, {5, 9, 0, 10})) std::printf("%d %d %d %d\n", t.src, t.walker, t.dst, t.copies);
  for (int r = 0; r < 4; ++r) {
    auto m = safire_b200::walker_moves(off, {5, 9, 0, 10}, r);
    std::printf("moves %d", r);
    for (auto* v : {&m.sends, &m.recvs, &m.copies}) {
      std::printf(" |");
      for (auto p : *v) std::printf(" %d %d", p.first, p.second);
    }
    std::printf("\n");
  }
  try {
    safire_b200::plan_walker_exchange(off, {5, 9});
  } catch (const safire_b200::Error& e) {
    std::printf("error %d\n", e.code);
  }
  return 0;
}
'''
    exe = str(tmp_path / "plan")
    r = subprocess.run([gxx, "-std=c++17", "-I", os.path.join(ROOT, "include"), "-x", "c++", "-", "-x", "none", lib,
                        "-o", exe, "-Wl,-rpath," + os.path.dirname(lib)], input=src, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0, out.stderr
    lines = out.stdout.strip().splitlines()
    w = np.array([0.0 if i % 5 == 0 else 0.25 * ((i * 7) % 11 + 1) for i in range(24)])
    off = O.comb(w, 0.3125, 24)
    assert [int(v) for v in lines[0].split()] == off.tolist()
    moves = [ln for ln in lines if ln.startswith("moves")]
    plan = [tuple(int(v) for v in ln.split()) for ln in lines[1:-1] if not ln.startswith("moves")]
    assert plan == O.plan_walker_exchange(off, [5, 9, 0, 10]) and plan
    for r, ln in enumerate(moves):
        parts = ln.split("|")[1:]
        got = [list(zip(*[iter(int(v) for v in p.split())] * 2)) for p in parts]
        assert got == [list(x) for x in O.walker_moves(off, [5, 9, 0, 10], r)]
    assert len(moves) == 4 and lines[-1] == "error 2"


def test_c_program_links_and_calls_the_host_entry_points(tmp_path):
    """include/safire_b200.h is valid C99 (-pedantic), and a C program linked against the library
    calls the host-only entry points (what a cgo or plain-C binding does) and agrees with the oracle."""
    import shutil
    import subprocess
    import numpy as np
    from oracle import afqmc_oracle as O
    from safire_b200 import build
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no gcc")
    lib = build.build()
    src = r'''
#include <stdio.h>
#include "safire_b200.h"
int main(void) {
  double w[12];
  int off[12], counts[3] = {4, 5, 3}, plan[4 * 15], n = 0, i;
  for (i = 0; i < 12; ++i) w[i] = (i == 2 || i == 9) ? 0.0 : 0.5 + 0.375 * ((i * 5) % 7);
  if (sfq_abi_version() != 13) return 3;
  if (sfq_comb_host(w, 0.71, 12, 12, off) != SFQ_OK) return 4;
  for (i = 0; i < 12; ++i) printf("%d ", off[i]);
  printf("\n");
  if (sfq_plan_walker_exchange(off, counts, 3, plan, 15, &n) != SFQ_OK) return 5;
  for (i = 0; i < n; ++i) printf("%d %d %d %d\n", plan[4 * i], plan[4 * i + 1], plan[4 * i + 2], plan[4 * i + 3]);
  if (sfq_plan_walker_exchange(off, counts, 3, plan, 0, &n) != SFQ_ERR_WORKSPACE || n == 0) return 6;
  printf("%s\n", sfq_last_error());
  {
    /* a rank's moves: exact room succeeds, one pair short reports the lengths and writes nothing */
    int sends[2 * 8], recvs[2 * 8], copies[2 * 8], ns = -1, nr = -1, nc = -1, r, ns2, nr2, nc2;
    for (r = 0; r < 3; ++r) {
      if (sfq_walker_moves(off, counts, 3, r, sends, 8, &ns, recvs, 8, &nr, copies, 8, &nc) != SFQ_OK) return 7;
      printf("moves %d %d %d %d\n", r, ns, nr, nc);
      if (ns > 0) {
        sends[0] = -7;
        if (sfq_walker_moves(off, counts, 3, r, sends, ns - 1, &ns2, recvs, 8, &nr2, copies, 8, &nc2) !=
                SFQ_ERR_WORKSPACE || ns2 != ns || nr2 != nr || nc2 != nc || sends[0] != -7)
          return 8;
      }
    }
  }
  return 0;
}
'''
    exe = str(tmp_path / "cplan")
    r = subprocess.run([gcc, "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I", os.path.join(ROOT, "include"),
                        "-x", "c", "-", "-x", "none", lib, "-o", exe, "-Wl,-rpath," + os.path.dirname(lib)],
                       input=src, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0, (out.returncode, out.stdout, out.stderr)
    lines = out.stdout.strip().splitlines()
    w = np.array([0.0 if i in (2, 9) else 0.5 + 0.375 * ((i * 5) % 7) for i in range(12)])
    off = O.comb(w, 0.71, 12)
    assert [int(v) for v in lines[0].split()] == off.tolist()
    moves = [ln for ln in lines if ln.startswith("moves")]
    lines = [ln for ln in lines if not ln.startswith("moves")]
    plan = [tuple(int(v) for v in ln.split()) for ln in lines[1:-1]]
    assert plan == O.plan_walker_exchange(off, [4, 5, 3]) and plan
    assert "room for 0" in lines[-1]
    assert len(moves) == 3
    for r, ln in enumerate(moves):
        s_, rv, cp = O.walker_moves(off, [4, 5, 3], r)
        assert [int(v) for v in ln.split()[1:]] == [r, len(s_), len(rv), len(cp)]
