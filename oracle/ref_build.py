"""Builds oracle/_ref/libref_pic.so from the reference's own source text.

TEST INFRASTRUCTURE ONLY.  The library built here is a checker of the
checker: CPU tests compare the oracle's restatement (pic_oracle.c) with the
reference's own code run on this machine.  Nothing in the CUDA library, the
GPU tests, smoke() or bench.py loads it.

The reference's particle kernels are SYCL (SYCL-PIC-poissonsolver/src/
mover.cpp, src/interpolation.cpp) and cannot be compiled here as files: no
SYCL compiler, no oneMKL.  The kernel bodies themselves are plain C++,
though.  This recipe reads them, unchanged, from a reference checkout:

  * modulo() and deterministic_mover()          src/mover.cpp:13-22, 103-176
  * the MoverKernel lambda                       src/mover.cpp:304-366
  * calculate_working_size() and the lambdas of
    PartialMeshInitKernel, InterpolationKernel,
    InterReductionKernel, ReducePartialMeshesKernel
    and RhoKernel, with the three set-up lines
    (denom, weighing, chrg) between them          src/interpolation.cpp:8-12, 39-171
  * Point / Field (include/point.hpp, included as is) and the GridParams
    struct (include/species_ds.hpp:6-10)

and wraps them in a host harness of its own: stand-ins for the few SYCL
names the bodies use (sycl::id, sycl::nd_item, sycl::atomic_ref), for the
hashmap's device view (retrieve / insert / deletion / key_idx / keys) and for
store_deleted_indices, plus serial loops in place of parallel_for.  The
generated translation unit goes to a temporary folder and is compiled with
the oracle's own flags (no FMA contraction: -march=x86-64-v2); only the shared
library lands in oracle/_ref/ (git-ignored).  No reference source is copied
into this repository.

    python oracle/ref_build.py [reference checkout root]   (default /root/reference)
"""
from __future__ import annotations

import os
import re
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
OUT = os.path.join(OUT_DIR, "libref_pic.so")
DEFAULT_ROOT = "/root/reference"
CXXFLAGS = ["-O3", "-march=x86-64-v2", "-fPIC", "-std=c++17", "-w"]


def _match_brace(text: str, open_at: int) -> int:
    """Index of the '}' closing the '{' at open_at, skipping comments and
    string / character literals."""
    assert text[open_at] == "{"
    depth, i, n = 0, open_at, len(text)
    while i < n:
        c = text[i]
        if text.startswith("//", i):
            i = text.find("\n", i)
            i = n if i < 0 else i
            continue
        if text.startswith("/*", i):
            i = text.index("*/", i) + 2
            continue
        if c in "\"'":
            j = i + 1
            while text[j] != c:
                j += 2 if text[j] == "\\" else 1
            i = j + 1
            continue
        if c == "{":
            depth += 1
        elif c == "}":
            depth -= 1
            if depth == 0:
                return i
        i += 1
    raise ValueError("unbalanced braces")


def _strip_comments_for_search(text: str) -> str:
    """Same length as text, with comments blanked (so that commented-out
    kernels are not found)."""
    out = list(text)
    i, n = 0, len(text)
    while i < n:
        if text.startswith("//", i):
            j = text.find("\n", i)
            j = n if j < 0 else j
            for k in range(i, j):
                out[k] = " "
            i = j
        elif text.startswith("/*", i):
            j = text.index("*/", i) + 2
            for k in range(i, j):
                if out[k] != "\n":
                    out[k] = " "
            i = j
        else:
            i += 1
    return "".join(out)


def function(text: str, head_regex: str) -> str:
    """A whole function definition, from its head to its closing brace."""
    live = _strip_comments_for_search(text)
    m = re.search(head_regex, live)
    if not m:
        raise ValueError(f"not found: {head_regex}")
    ob = live.index("{", m.end())
    return text[m.start():_match_brace(text, ob) + 1]


def kernel_lambda(text: str, kernel: str) -> tuple[str, str]:
    """(parameter declaration, body) of the lambda passed to
    parallel_for<kernel> (the live, uncommented one)."""
    live = _strip_comments_for_search(text)
    m = re.search(r"parallel_for<\s*" + re.escape(kernel) + r"\s*>\s*\(", live)
    if not m:
        raise ValueError(f"kernel {kernel} not found")
    lm = re.compile(r"\[=\]\s*\(([^)]*)\)\s*\{").search(live, m.end())
    ob = lm.end() - 1
    cb = _match_brace(text, ob)
    return lm.group(1).strip(), text[ob + 1:cb]


def statement(text: str, regex: str) -> str:
    live = _strip_comments_for_search(text)
    m = re.search(regex, live)
    if not m:
        raise ValueError(f"statement not found: {regex}")
    return text[m.start():m.end()]


HARNESS_HEAD = r"""
// Generated by oracle/ref_build.py from the reference's source text; not
// committed.  Harness code (everything outside the marked extracts) is the
// repository's own.
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <vector>
#include <math.h>

namespace sycl {
enum class memory_order { relaxed, acq_rel };
enum class memory_scope { device };
namespace access { enum class address_space { global_space }; }
// Serial loops: a plain read-modify-write is the atomic.
template <class T, memory_order O, memory_scope S, access::address_space A>
struct atomic_ref {
    T& r;
    explicit atomic_ref(T& x) : r(x) {}
    T fetch_add(T v) const { T o = r; r += v; return o; }
    T load() const { return r; }
};
template <int D> struct id {
    size_t v;
    explicit id(size_t x) : v(x) {}
    operator size_t() const { return v; }
    size_t operator[](int) const { return v; }
};
template <int D> struct nd_item {
    size_t g, l;
    size_t get_global_id(int) const { return g; }
    size_t get_local_id(int) const { return l; }
};
}  // namespace sycl
"""

HARNESS_MAP = r"""
// Stand-in for sycl_hashmap::DeviceView.  Buckets are rows of probing_length
// slots (bucket key * probing_length), keys[slot] = 1 for a used slot,
// values[slot] = particle index.  insert() and deletion() only record what
// the mover asked for: the bucket a particle is inserted into (returned as
// its new pointer) and the slots deleted.
struct HarnessMap {
    int* keys;
    int* values;
    int capacity;
    int probing_length;
    int* key_idx;
    int* delete_idx;
    int* inserted_key;   // per particle index: bucket of the insert, or -1
    int* deleted_slot;   // per particle index: the slot deleted, or -1
    int* retrieve(int key) const {
        const int idx = key * probing_length;
        if (idx >= capacity) return NULL;
        return values + idx;
    }
    int insert(int key, int value, int* NUM_Points) const {
        (void)NUM_Points;
        inserted_key[value] = key;
        return key;
    }
    void deletion(int key, int* NUM_Points) const {
        (void)NUM_Points;
        deleted_slot[key] = key;
    }
};

// store_deleted_indices (include/utils.hpp:45-56) appends an index to a list
// with an atomic counter, up to n entries.
inline int store_deleted_indices(int index, int* empty_space, int* empty_space_count, int n) {
    const int k = (*empty_space_count)++;
    if (k < n) {
        empty_space[k] = index;
        return 1;
    }
    return 0;
}
"""


def generate(root: str) -> str:
    sp = os.path.join(root, "SYCL-PIC-poissonsolver")
    mover = open(os.path.join(sp, "src", "mover.cpp")).read()
    interp = open(os.path.join(sp, "src", "interpolation.cpp")).read()
    species = open(os.path.join(sp, "include", "species_ds.hpp")).read()
    gridparams = statement(species, r"struct\s+GridParams\s*\{[^}]*\};")
    f_modulo = function(mover, r"double\s+modulo\s*\(\s*double\s+x\s*,\s*double\s+y\s*\)")
    f_mover = function(mover, r"inline\s+void\s+deterministic_mover\s*\(")
    mv_par, mv_body = kernel_lambda(mover, "MoverKernel")
    f_ws = function(interp, r"int\s+calculate_working_size\s*\(")
    init_par, init_body = kernel_lambda(interp, "PartialMeshInitKernel")
    ik_par, ik_body = kernel_lambda(interp, "InterpolationKernel")
    red_par, red_body = kernel_lambda(interp, "InterReductionKernel")
    pm_par, pm_body = kernel_lambda(interp, "ReducePartialMeshesKernel")
    rho_par, rho_body = kernel_lambda(interp, "RhoKernel")
    s_denom = statement(interp, r"const\s+double\s+denom\s*=[^;]*;")
    s_weigh = statement(interp, r"const\s+double\s+weighing\s*=\s*weighingFactor\[ptype\]\s*;")
    s_chrg = statement(interp, r"double\s+chrg\s*=\s*-particleCharges\[ptype\]\s*/\s*epsilon\s*;")
    for par in (mv_par, init_par, red_par, pm_par, rho_par):
        assert par.startswith("sycl::id<1>"), par
    assert ik_par.startswith("sycl::nd_item<1>"), ik_par
    mv_var, init_var = mv_par.split()[-1], init_par.split()[-1]
    ik_var, red_var = ik_par.split()[-1], red_par.split()[-1]
    pm_var, rho_var = pm_par.split()[-1], rho_par.split()[-1]

    src = [HARNESS_HEAD,
           f'#include "{os.path.join(sp, "include", "point.hpp")}"\n',
           "// ---- extract: include/species_ds.hpp GridParams\n", gridparams, "\n",
           HARNESS_MAP,
           "// ---- extract: src/mover.cpp modulo\n", f_modulo, "\n",
           "// ---- extract: src/mover.cpp deterministic_mover\n", f_mover, "\n",
           "// ---- extract: src/interpolation.cpp calculate_working_size\n", f_ws, "\n"]

    src.append(r"""
// MoverKernel over num_particles Points, serially in index order.  Outputs:
// the Points as the kernel leaves them (pointer -1: deleted; otherwise the
// bucket it was re-inserted into, or its old pointer when it stayed), the
// left-exit count (new_additions) and the number of holes recorded.
extern "C" int ref_mover_kernel(Point* points_device, int num_particles, const GridParams* gp,
                                const double* CtoM, int ptype, double dt, const Field* electricField,
                                const double* magneticField, const double* phi, int periodicBoundary,
                                int* inserted_key, int* deleted_slot, int* left_exits) {
    const GridParams params = *gp;
    const int periodicBoundary_local = periodicBoundary;
    const double* CtoM_local = CtoM;
    const double dt_local = dt;
    const Field* electric_field_local = electricField;
    const double* magnetic_field_local = magneticField;
    const double* phi_local = phi;
    HarnessMap dmap{nullptr, nullptr, 0, 0, nullptr, nullptr, inserted_key, deleted_slot};
    int num_points_v = 0;
    int* NUM_Points = &num_points_v;
    std::vector<int> empty_v(num_particles + 1), left_v(num_particles + 1);
    int empty_n = 0, left_n = 0, err = 0, adds = 0;
    int* empty_space = empty_v.data();
    int* empty_space_idx = &empty_n;
    int* mover_left_local = left_v.data();
    int* mover_idx_local = &left_n;
    int* error_flag = &err;
    int* new_additions = &adds;
    for (int i = 0; i < num_particles; ++i) { inserted_key[i] = -1; deleted_slot[i] = -1; }
    auto kernel = [=](""" + mv_par + ") {\n// ---- extract: src/mover.cpp MoverKernel body\n" + mv_body + r"""
    };
    for (int i = 0; i < num_particles; ++i) kernel(sycl::id<1>((size_t)i));
    *left_exits = adds;
    return empty_n;
}

// interpolate() (src/interpolation.cpp:13-171) for one species on a harness
// hashmap: particles are placed into their buckets in index order
// (key = bucket_key[i], -1 = absent), probing_length slots a bucket.
extern "C" int ref_interpolate(const Point* points_device, int n, const int* bucket_key,
                               const GridParams* gp, int probing_length, int prob_size,
                               const double* CtoM, const double* weighingFactor,
                               const double* particleCharges, double epsilon, int ptype,
                               double* final_mesh, double* energy_mesh, double* rho) {
    const GridParams params = *gp;
    const size_t gridSize = static_cast<size_t>(params.GRID_X) * params.GRID_Y;
    const int capacity = (int)(gridSize * probing_length);
    std::vector<int> keys_v(capacity, 0), values_v(capacity, -1), key_idx_v(gridSize, 0);
    for (int i = 0; i < n; ++i) {
        const int k = bucket_key[i];
        if (k < 0) continue;
        if (key_idx_v[k] >= probing_length) return -1;
        const int slot = k * probing_length + key_idx_v[k]++;
        keys_v[slot] = 1;
        values_v[slot] = i;
    }
    std::vector<int> none(n > 0 ? n : 1, -1);
    HarnessMap dmap{keys_v.data(), values_v.data(), capacity, probing_length, key_idx_v.data(),
                    nullptr, none.data(), none.data()};
    std::vector<double> cm(4 * gridSize), cme(4 * gridSize);
    std::vector<double> acc(8 * gridSize * (size_t)prob_size);
    double* corner_mesh = cm.data();
    double* corner_mesh_enrgy = cme.data();
    double* accessor_s1 = acc.data();
    double* accessor_s2 = accessor_s1 + gridSize * prob_size;
    double* accessor_s3 = accessor_s2 + gridSize * prob_size;
    double* accessor_s4 = accessor_s3 + gridSize * prob_size;
    double* accessor_s1_enrgy = accessor_s4 + gridSize * prob_size;
    double* accessor_s2_enrgy = accessor_s1_enrgy + gridSize * prob_size;
    double* accessor_s3_enrgy = accessor_s2_enrgy + gridSize * prob_size;
    double* accessor_s4_enrgy = accessor_s3_enrgy + gridSize * prob_size;
    {
        auto k0 = [=](""" + init_par + ") {\n// ---- extract: PartialMeshInitKernel body\n" + init_body + r"""
        };
        for (size_t i = 0; i < 4 * gridSize; ++i) k0(sycl::id<1>(i));
    }
    size_t global_size = gridSize * prob_size;
    // ---- extract: set-up lines
    """ + s_denom + "\n    " + s_weigh + r"""
    {
        auto k1 = [=](""" + ik_par + ") {\n// ---- extract: InterpolationKernel body\n" + ik_body + r"""
        };
        for (size_t g = 0; g < global_size; ++g) k1(sycl::nd_item<1>{g, g % (size_t)prob_size});
    }
    {
        auto k2 = [=](""" + red_par + ") {\n// ---- extract: InterReductionKernel body\n" + red_body + r"""
        };
        for (size_t i = 0; i < gridSize; ++i) k2(sycl::id<1>(i));
    }
    {
        auto k3 = [=](""" + pm_par + ") {\n// ---- extract: ReducePartialMeshesKernel body\n" + pm_body + r"""
        };
        for (size_t i = 0; i < gridSize; ++i) k3(sycl::id<1>(i));
    }
    """ + s_chrg + r"""
    {
        auto k4 = [=](""" + rho_par + ") {\n// ---- extract: RhoKernel body\n" + rho_body + r"""
        };
        for (size_t i = 0; i < gridSize; ++i) k4(sycl::id<1>(i));
    }
    return 0;
}
""")
    return "".join(src)


def build(root: str | None = None, quiet: bool = True) -> str:
    """Generates the harness from the reference checkout at `root` and
    compiles it into oracle/_ref/libref_pic.so; returns that path."""
    root = root or os.environ.get("PIC_REFERENCE_ROOT", DEFAULT_ROOT)
    if not os.path.isdir(os.path.join(root, "SYCL-PIC-poissonsolver", "src")):
        raise FileNotFoundError(f"no SYCL-PIC-poissonsolver sources under {root}")
    os.makedirs(OUT_DIR, exist_ok=True)
    with tempfile.TemporaryDirectory() as tmp:
        cpp = os.path.join(tmp, "ref_pic.cpp")
        with open(cpp, "w") as f:
            f.write(generate(root))
        tmp_so = os.path.join(tmp, "libref_pic.so")
        subprocess.run(["g++", *CXXFLAGS, "-shared", "-o", tmp_so, cpp, "-lm"], check=True,
                       stdout=subprocess.DEVNULL if quiet else None)
        shutil.move(tmp_so, OUT + ".tmp")
        os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(sys.argv[1] if len(sys.argv) > 1 else None, quiet=False))
