"""Build libbgp.so in-tree for sm_100a.

One translation unit per compiled grid size (N, M) keeps every kernel small
enough for ptxas and lets the sizes compile in parallel; a generated header
lists the sizes for the host dispatcher. Objects are rebuilt only when a
source or header is newer.

    python -m becgpp_b200.build [-j JOBS] [--force] [--profile]

--profile builds a second library, libbgp_prof.so, from the same sources with
the phase profiler compiled in (-DBGP_PROF): thread 0 of every team's first CTA
accumulates, per kind of phase, the time spent working, reducing, waiting at
the team barrier and gathering the reduced values. Select it at run time with
BECGPP_B200_LIB=<path>; `python bench.py --case phases` does so and prints the
breakdown.
"""
import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(os.path.dirname(HERE), "_build", "bgp")
GEN = os.path.join(BUILD, "gen")
LIB = os.path.join(HERE, "libbgp.so")
PROF_LIB = os.path.join(HERE, "libbgp_prof.so")

# grid sizes compiled into the solver: N per axis, M = 2N with a long-range kernel
SIZES_N = (16, 24, 32, 48, 64, 96, 128, 192, 256, 384, 512)
MAX_N_WITH_KERNEL = 384
# two-size kernels for batches that mix grids (sweeps over 128^2 and 256^2)
COMBOS = ((128, 0, 256, 0),)

# stream-pass candidates of the autotuner: radix orders of the line FFT and lines
# per tile (a strided tile groups that many neighbours, so N must be a multiple;
# the tile must fit in shared memory)
RADIX_ORDERS = (0, 1, 2)   # Stockham stage orders; 3 = the register-resident transform (N = 32 R)
CONV_LINES = (1, 2, 4, 8, 16)


def radix_orders(n):
    """Transforms of the stream H psi passes: 0-2 Stockham orders, 3 the register
    transform (N = 32 R); each again at doubled occupancy (+4: half the registers)."""
    base = RADIX_ORDERS + ((3,) if n % 32 == 0 else ())
    return base + tuple(v + 4 for v in base)


def stream_lines(n):
    def smem(L, ln):
        pitch = ((L + L // 8 + 1) | 1) if ln >= 8 else (((L + L // 8 + 1 + 5) // 8) * 8 + 2)
        return ln * pitch * 16
    return [ln for ln in (1, 2, 4, 8, 16) if n % ln == 0 and ln <= n and smem(n, ln) <= 160 * 1024]


def conv_lines(m):
    """Lines per tile of the stream convolution passes over the padded length m:
    the line buffers and the tile's kernel slab must fit in shared memory."""
    def smem(L, ln):
        pitch = ((L + L // 8 + 1) | 1) if ln >= 8 else (((L + L // 8 + 1 + 5) // 8) * 8 + 2)
        slab = ((ln * ((L // 2 + 1) | 1) * 8 + 15) // 16) * 16
        return ln * pitch * 16 + slab
    return [ln for ln in CONV_LINES if smem(m, ln) <= 200 * 1024]


NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2"]


def pairs():
    out = []
    for n in SIZES_N:
        out.append((n, 0))
        if n <= MAX_N_WITH_KERNEL:
            out.append((n, 2 * n))
    return out


def _write_if_changed(path, text):
    if os.path.isfile(path) and open(path).read() == text:
        return
    with open(path, "w") as f:
        f.write(text)


def generate():
    os.makedirs(GEN, exist_ok=True)
    units = []
    hdr = ["// generated by becgpp_b200/build.py: compiled grid sizes", "#pragma once"]
    hdr.append("#define BGP_FOR_SIZES(X) " + " ".join(f"X({n}, {m})" for n, m in pairs()))
    hdr.append("#define BGP_FOR_COMBOS(X) " + " ".join(f"X({a}, {b}, {c}, {d})" for a, b, c, d in COMBOS))
    hdr.append("#define BGP_FOR_TABLE_LENGTHS(X) "
               + " ".join(f"X({m})" for m in sorted({m for _, m in pairs() if m})))
    # each kernel per grid dimension (BGP_NDIM) and twice: FP64 only, and with the
    # FP32 transforms of the mixed form (BGP_MIXED=1, symbols suffixed _mx)
    for sfx, mixed in (("", 0), ("_mx", 1)):
        for dim in (2, 3):
            pre = f"#define BGP_MIXED {mixed}\n#define BGP_NDIM {dim}\n"
            for n, m in pairs():
                name = f"{n}_{m}_d{dim}{sfx}"
                hdr.append(f'extern "C" void* bgp_kptr_{name}();')
                src = (pre + f'#include "bgp_kernel.cuh"\n'
                       f"template __global__ void bgp::bgp_kernel_t<{n}, {m}>(bgp::Launch);\n"
                       f'extern "C" void* bgp_kptr_{name}() {{ return (void*)&bgp::bgp_kernel_t<{n}, {m}>; }}\n')
                path = os.path.join(GEN, f"k_{name}.cu")
                _write_if_changed(path, src)
                units.append(path)
            if dim != 2:
                continue   # the two-size kernels serve 2D batches
            for a, b, c, d in COMBOS:
                name = f"{a}_{b}_{c}_{d}_d{dim}{sfx}"
                hdr.append(f'extern "C" void* bgp_kptr2_{name}();')
                src = (pre + f'#include "bgp_kernel.cuh"\n'
                       f"template __global__ void bgp::bgp_kernel_t2<{a}, {b}, {c}, {d}>(bgp::Launch);\n"
                       f'extern "C" void* bgp_kptr2_{name}() '
                       f"{{ return (void*)&bgp::bgp_kernel_t2<{a}, {b}, {c}, {d}>; }}\n")
                path = os.path.join(GEN, f"k2_{name}.cu")
                _write_if_changed(path, src)
                units.append(path)
    # stream passes (standalone and batched H psi): one unit per line length N with
    # every (lines per tile, radix order) candidate of the autotuner, and the
    # convolution passes of the padded length M = 2N
    hdr.append("#define BGP_FOR_STREAM_N(X) " + " ".join(f"X({n})" for n in SIZES_N))
    hdr.append("#define BGP_FOR_STREAM_M(X) " + " ".join(f"X({2 * n})" for n in SIZES_N if n <= MAX_N_WITH_KERNEL))
    for n in SIZES_N:
        lns = stream_lines(n)
        hdr.append(f'extern "C" void* bgp_sptr_{n}(int ln, int v);')
        lines = ['#include "bgp_stream.cuh"']
        cases = []
        for ln in lns:
            for v in radix_orders(n):
                lines.append(f"template __global__ void bgp::k_stream_h<{n}, {ln}, {v}>(bgp::SLaunch, int, int);")
                cases.append(f"  if (ln == {ln} && v == {v}) return (void*)&bgp::k_stream_h<{n}, {ln}, {v}>;")
        lines.append(f'extern "C" void* bgp_sptr_{n}(int ln, int v) {{')
        lines += cases
        lines.append("  return nullptr;\n}")
        if n <= MAX_N_WITH_KERNEL:
            m = 2 * n
            hdr.append(f'extern "C" void* bgp_scptr_{m}(int ln, int v);')
            ccases = []
            for ln in conv_lines(m):
                for v in (0, 3) if m % 32 == 0 else (0,):
                    lines.append(f"template __global__ void bgp::k_stream_conv<{m}, {ln}, {v}>(bgp::SLaunch, int);")
                    ccases.append(f"  if (ln == {ln} && v == {v}) return (void*)&bgp::k_stream_conv<{m}, {ln}, {v}>;")
            lines.append(f'extern "C" void* bgp_scptr_{m}(int ln, int v) {{')
            lines += ccases
            lines.append("  return nullptr;\n}")
        path = os.path.join(GEN, f"s_{n}.cu")
        _write_if_changed(path, "\n".join(lines) + "\n")
        units.append(path)
    _write_if_changed(os.path.join(GEN, "bgp_sizes_gen.h"), "\n".join(hdr) + "\n")
    return units


# headers the persistent solver kernels include (the generated per-size units);
# the host units (bgp_api.cu, bgp_noalloc.cu, bgp_diag.cu, bgp_vortex.cu) depend on every header
KERNEL_HEADERS = ("bgp_kernel.cuh", "bgp_programs.cuh", "bgp_passes.cuh", "bgp_device.cuh", "bgp_fft.cuh",
                  "bgp_common.cuh")


def _deps(src):
    # (the generated unit itself carries its instantiations, so build.py is no dependency)
    if os.path.basename(src).startswith(("k_", "k2_")):
        return [os.path.join(CSRC, f) for f in KERNEL_HEADERS]
    if os.path.basename(src).startswith("s_"):
        return [os.path.join(CSRC, f) for f in KERNEL_HEADERS + ("bgp_stream.cuh", "bgp_regfft.cuh")]
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".cu", ".h"))] + [
        os.path.join(os.path.dirname(HERE), "include", "bgp.h"), os.path.abspath(__file__)]


def _compile(src, obj, force):
    newest = max(os.path.getmtime(p) for p in _deps(src) + [src])
    if not force and os.path.isfile(obj) and os.path.getmtime(obj) >= newest:
        return obj, None
    cmd = [NVCC, *ARCH, *FLAGS, "-I", CSRC, "-I", GEN, "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, f"{' '.join(cmd)}\n{r.stdout}\n{r.stderr}"
    return obj, None


def build(jobs=None, force=False, verbose=True):
    units = generate()
    units.append(os.path.join(CSRC, "bgp_api.cu"))
    units.append(os.path.join(CSRC, "bgp_noalloc.cu"))
    units.append(os.path.join(CSRC, "bgp_diag.cu"))
    units.append(os.path.join(CSRC, "bgp_vortex.cu"))
    os.makedirs(BUILD, exist_ok=True)
    objs = [os.path.join(BUILD, os.path.splitext(os.path.basename(u))[0] + ".o") for u in units]
    jobs = jobs or max(1, os.cpu_count() or 1)
    errors = []
    with cf.ThreadPoolExecutor(jobs) as ex:
        futs = [ex.submit(_compile, u, o, force) for u, o in zip(units, objs)]
        for f in cf.as_completed(futs):
            obj, err = f.result()
            if err:
                errors.append(err)
            elif verbose:
                print(f"[build] {os.path.basename(obj)}", flush=True)
    if errors:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errors))
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.isfile(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    if verbose:
        print(f"[build] {LIB}", flush=True)
    return LIB


def build_profiler(jobs=None, force=False, verbose=True, sizes=None):
    """libbgp_prof.so: the same library with the phase profiler compiled in
    (optionally only the grid sizes N in `sizes`)."""
    global BUILD, GEN, LIB, FLAGS, SIZES_N
    saved = BUILD, GEN, LIB, FLAGS, SIZES_N
    BUILD = os.path.join(os.path.dirname(HERE), "_build", "bgp_prof")
    GEN = os.path.join(BUILD, "gen")
    LIB = PROF_LIB
    FLAGS = FLAGS + ["-DBGP_PROF"]
    if sizes:
        SIZES_N = tuple(sizes)
    try:
        return build(jobs, force, verbose)
    finally:
        BUILD, GEN, LIB, FLAGS, SIZES_N = saved


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("-j", "--jobs", type=int, default=None)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--profile", action="store_true", help="build libbgp_prof.so (phase profiler)")
    ap.add_argument("--sizes", default=None, help="--profile: comma-separated grid sizes N to compile")
    a = ap.parse_args()
    try:
        if a.profile:
            build_profiler(a.jobs, a.force, sizes=[int(x) for x in a.sizes.split(",")] if a.sizes else None)
        else:
            build(a.jobs, a.force)
    except RuntimeError as e:
        print(e, file=sys.stderr)
        sys.exit(1)
