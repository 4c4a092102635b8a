"""The device headers compile under NVRTC without host headers.

Generic tables are compiled at run time (csrc/rtc.cu): the source includes
k_generic_tma.cuh, which pulls in device.cuh and views.h, and the library
hands NVRTC only a prelude of fixed-width types, the tensor-map type and two
macros. These tests compile programs of the generated shape for float and
double on the CPU (NVRTC needs no GPU), so a host-only include or construct
slipping into those headers fails here rather than on the GPU, where the
library would quietly fall back to the interpreting kernel.
"""
import os

import pytest

nvrtc = pytest.importorskip("cuda.bindings.nvrtc")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "physis_b200", "csrc")

PRELUDE = """
typedef signed char int8_t; typedef unsigned char uint8_t;
typedef short int16_t; typedef unsigned short uint16_t;
typedef int int32_t; typedef unsigned int uint32_t;
typedef long long int64_t; typedef unsigned long long uint64_t;
typedef unsigned long size_t; typedef unsigned long uintptr_t;
struct __align__(64) CUtensorMap_st { unsigned long long opaque[16]; };
typedef CUtensorMap_st CUtensorMap;
#define PSB_MAX_TERMS 32
#define PSB_MAX_GRIDS 16
"""

# A term program of the generated shape: a run of three terms on one row
# (x offsets -1, 0, +1, the middle one unmultiplied), then a run of one term
# on another plane, then the first term of a third row.
PROGRAM = r"""
#include "k_generic_tma.cuh"
namespace psb {
struct GtCompiledProg {
  static constexpr bool kCompiled = true;
  static constexpr bool kPoints = false;
  template <typename T>
  static __device__ __forceinline__ void eval(const GtTable &tab, const unsigned char *ring,
      int sbytes, int S, int slot0, int thr_off, int bx, int lane, GtBlk<T> &acc) {
    GtRow<T> row[kGtVY];
    gt_rows<T>(ring, sbytes, S, slot0, thr_off, bx, lane, 0, -136, true, true, row);
    gt_term<1, false, true>(row, gt_coef(tab, 0, T()), acc);
    gt_term<2, true, false>(row, gt_coef(tab, 1, T()), acc);
    gt_term<3, false, false>(row, gt_coef(tab, 2, T()), acc);
    gt_rows<T>(ring, sbytes, S, slot0, thr_off, bx, lane, 2, 136, false, true, row);
    gt_term<0, false, false>(row, gt_coef(tab, 3, T()), acc);
    gt_rows<T>(ring, sbytes, S, slot0, thr_off, bx, lane, 1, 0, true, false, row);
    gt_term<4, false, false>(row, gt_coef(tab, 4, T()), acc);
  }
};
}  // namespace psb
extern "C" __global__ void __launch_bounds__(psb::kGtThreads, MINB)
psb_generic_tma_compiled(const __grid_constant__ psb::GtMaps maps,
                         const __grid_constant__ psb::GtTable tab, psb::GridView out,
                         psb::Dom3 d, const __grid_constant__ psb::GtGeom geo, int *err) {
  psb::gt_body<TYPE, psb::GtCompiledProg>(maps, tab, out, d, geo, err);
}
"""


# A general program: products of two reads, a constant times a read, a bare
# read.
GENERAL = r"""
#include "k_generic_tma.cuh"
namespace psb {
struct GtCompiledProg {
  static constexpr bool kCompiled = true;
  static constexpr bool kPoints = false;
  template <typename T>
  static __device__ __forceinline__ void eval(const GtTable &tab, const unsigned char *ring,
      int sbytes, int S, int slot0, int thr_off, int bx, int lane, GtBlk<T> &acc) {
    (void)lane;
    gt_general_term<T>(GtFactor{2, 1, -140, 0, tab.a[0].c}, GtFactor{2, 0, 2880, 0, tab.b[0].c},
                       true, ring, sbytes, S, slot0, thr_off, bx, acc);
    gt_general_term<T>(GtFactor{0, 0, 0, 0, tab.a[1].c}, GtFactor{2, 2, 5, 0, tab.b[1].c},
                       false, ring, sbytes, S, slot0, thr_off, bx, acc);
    gt_general_term<T>(GtFactor{2, 1, 0, 0, tab.a[2].c}, GtFactor{1, 0, 0, 0, tab.b[2].c},
                       false, ring, sbytes, S, slot0, thr_off, bx, acc);
  }
};
}  // namespace psb
extern "C" __global__ void __launch_bounds__(psb::kGtThreads, MINB)
psb_generic_tma_compiled(const __grid_constant__ psb::GtMaps maps,
                         const __grid_constant__ psb::GtTable tab, psb::GridView out,
                         psb::Dom3 d, const __grid_constant__ psb::GtGeom geo, int *err) {
  psb::gt_body<TYPE, psb::GtCompiledProg>(maps, tab, out, d, geo, err);
}
"""


def _compile(src, opts):
    err, prog = nvrtc.nvrtcCreateProgram(src.encode(), b"psb_stencil.cu", 1, [PRELUDE.encode()],
                                         [b"psb_rtc_prelude.h"])
    assert err == nvrtc.nvrtcResult.NVRTC_SUCCESS
    res = nvrtc.nvrtcCompileProgram(prog, len(opts), [o.encode() for o in opts])[0]
    _, n = nvrtc.nvrtcGetProgramLogSize(prog)
    log = b" " * n
    nvrtc.nvrtcGetProgramLog(prog, log)
    size = 0
    if res == nvrtc.nvrtcResult.NVRTC_SUCCESS:
        _, size = nvrtc.nvrtcGetCUBINSize(prog)
    nvrtc.nvrtcDestroyProgram(prog)
    return res, log.decode(errors="replace"), size


@pytest.mark.parametrize("typ,minb", [("float", 4), ("double", 3)])
@pytest.mark.parametrize("packed_mul", [0, 1, 2])
def test_generated_kernel_compiles_for_sm100a(typ, minb, packed_mul):
    src = PROGRAM.replace("MINB", str(minb)).replace("TYPE", typ)
    opts = ["--gpu-architecture=sm_100a", "-std=c++17", "--fmad=false", "-default-device",
            "-I" + CSRC, "-DPSB_GT_VY=4", "-DPSB_GT_PACKED_MUL=%d" % packed_mul]
    res, log, size = _compile(src, opts)
    assert res == nvrtc.nvrtcResult.NVRTC_SUCCESS, log
    assert size > 0


@pytest.mark.parametrize("typ,minb", [("float", 4), ("double", 3)])
def test_generated_general_kernel_compiles_for_sm100a(typ, minb):
    src = GENERAL.replace("MINB", str(minb)).replace("TYPE", typ)
    opts = ["--gpu-architecture=sm_100a", "-std=c++17", "--fmad=false", "-default-device",
            "-I" + CSRC, "-DPSB_GT_VY=4"]
    res, log, size = _compile(src, opts)
    assert res == nvrtc.nvrtcResult.NVRTC_SUCCESS, log
    assert size > 0


def test_prelude_matches_the_library():
    """The test's prelude is the one csrc/rtc.cu builds (same types, same
    macro values as the public header)."""
    with open(os.path.join(CSRC, "rtc.cu")) as f:
        rtc = f.read()
    for line in ("typedef long long int64_t;", "typedef unsigned long long uint64_t;",
                 "struct __align__(64) CUtensorMap_st { unsigned long long opaque[16]; };"):
        assert line in rtc.replace("\\n", "\n"), line
    with open(os.path.join(ROOT, "include", "physis_b200.h")) as f:
        hdr = f.read()
    assert "#define PSB_MAX_TERMS 32" in hdr and "#define PSB_MAX_GRIDS 16" in hdr
