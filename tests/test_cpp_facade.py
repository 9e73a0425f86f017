"""The C++ boundary compiles as a caller of the reference would use it (CPU):

* tests/cpp/facade_check.cpp against the C++23 facade include/iceicle_b200.hpp
  (the reference's concept-shaped flux objects, ConservationLawDDG,
  form_residual, form_jacobian_fd, NewtonSolver), compiled with g++ -std=c++23
  and linked against the product library; its run on a GPU is
  tests/test_gpu_cpp_facade.py;
* every C++ call site shown in INTEGRATION.md, compiled (g++ -std=c++23
  -fsyntax-only) inside one function after a prelude that declares the
  reference-side objects the snippets name (mesh, disc, coeffs, conv, ...)."""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA_INC = "/usr/local/cuda/include"
LIB = os.path.join(ROOT, "iceicle_b200", "libiceicle_b200.so")

needs_gxx = pytest.mark.skipif(shutil.which("g++") is None or not os.path.isdir(CUDA_INC),
                               reason="g++ or the CUDA headers absent")


def build_facade_check(out):
    cmd = ["g++", "-std=c++23", "-O1", "-Wall", "-I", os.path.join(ROOT, "include"), "-I", CUDA_INC,
           os.path.join(ROOT, "tests", "cpp", "facade_check.cpp"), "-o", out,
           "-L", os.path.dirname(LIB), "-liceicle_b200", "-L", "/usr/local/cuda/lib64", "-lcudart",
           f"-Wl,-rpath,{os.path.dirname(LIB)}"]
    return subprocess.run(cmd, capture_output=True, text=True)


@needs_gxx
@pytest.mark.skipif(not os.path.exists(LIB), reason="product library not built")
def test_facade_program_compiles_and_links(tmp_path):
    r = build_facade_check(str(tmp_path / "facade_check"))
    assert r.returncode == 0, r.stderr[-4000:]


PRELUDE = r'''
#include <array>
#include <functional>
#include <vector>
#include "iceicle_b200.h"
#include "iceicle_b200.hpp"
// the reference-side objects the call sites name (shapes as in the reference)
struct Coeffs { double mu; std::array<double, 2> a, b; };
struct Disc { bool interior_penalty; double sigma_ic;
              std::vector<std::function<void(const double*, double*)>> dirichlet_callbacks; };
struct Mesh { std::vector<std::array<double, 2>> coord; };
struct Conv { double tau_abs, tau_rel; int kmax; };
void integration_call_sites(icx_ctx* ctx_past, icx_ctx** parts, int n_parts, double* d_u, double* d_res,
                            double* d_bsr_vals, double* d_u_all, double* d_u_past, double* d_vals, double* d_x,
                            double* d_samples, double* d_res_and_ic, void* stream) {
  int nx = 8, ny = 8, geometry_order = 2, basis_order = 2, p = 2, cap = 16, ns = 0, it = 0, k = 1, itime = 0;
  long long n_dof = 0;
  double rr = 0.0, tfinal = 1.0, mu = 0.01, T0 = 0.004, T1 = 0.005, rho_inf = 1.0, u_inf = 0.5, T_inf = 0.004;
  double* d_y = d_x;
  float* d_vals32 = nullptr;
  double* d_u_set = d_u_all;
  double mu_ratio = 0.02, T0_ratio = 0.004, Ts_ratio = 0.0015;
  std::vector<int> groups_v(64, 0);
  const int* groups = groups_v.data();
  Coeffs coeffs{0.01, {0.0, 0.0}, {1.0, 0.5}}, c = coeffs;
  Disc disc{false, 0.0, {}};
  disc.dirichlet_callbacks.push_back([](const double*, double* out) { out[0] = 0.0; });
  Mesh mesh{std::vector<std::array<double, 2>>(289)};
  Conv conv{1e-10, 0.0, 20};
  std::vector<int> traces{0, 1, 2};
  (void)n_dof; (void)ns; (void)it; (void)rr;
'''


@needs_gxx
def test_integration_md_call_sites_compile(tmp_path):
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    blocks = re.findall(r"```cpp\n(.*?)```", text, flags=re.S)
    assert len(blocks) >= 2
    # the facade example is self-contained: its own scope (its names repeat the reference-side ones)
    body = "\n".join(("{\n" + b.replace('#include "iceicle_b200.hpp"', "") + "\n}") if "iceicle_b200.hpp" in b
                     else b.replace('#include "iceicle_b200.h"', "") for b in blocks)
    src = tmp_path / "call_sites.cpp"
    src.write_text(PRELUDE + body + "\n}\n")
    r = subprocess.run(["g++", "-std=c++23", "-fsyntax-only", "-Wno-unused-variable", "-I",
                        os.path.join(ROOT, "include"), "-I", CUDA_INC, str(src)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
