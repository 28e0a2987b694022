"""CPU tests of the shader harness's own parts (oracle/glsl/extract.py and
oracle/glsl/glsl.h), independent of the reference tree: a small GLSL stage
written here is cut out, translated, compiled against glsl.h with g++ and run,
and its outputs are checked against the rules the harness states (literal
types, block and interface translation, swizzle reads and writes, left-to-right
products, mix / clamp / fract definitions, saturating conversions, discard,
shared arrays with barriers)."""
from __future__ import annotations

import shutil
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "oracle" / "glsl"))

import extract  # noqa: E402

pytestmark = pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")

STAGES = """\
// a test shader in the sokol-shdc layout
@cs probe_cs
struct Item {
    vec4 a;
    uvec2 u;
};

layout(binding = 0) uniform ProbeUBO {
    mat4 m;
    vec2 scale;
    int count;
    float t;
};

layout(binding = 1) buffer Items {
    Item items[];
};

layout(binding = 2) readonly buffer Inputs {
    float inputs[];
};

shared uint partial[4];

layout(local_size_x = 4, local_size_y = 1, local_size_z = 1) in;

void main() {
    uint lid = gl_LocalInvocationID.x;
    partial[lid] = uint(inputs[lid] * 2.5);
    barrier();
    uint total = partial[0] + partial[1] + partial[2] + partial[3];
    int k = int(gl_GlobalInvocationID.x);
    if (k >= count) return;
    vec4 p = m * vec4(inputs[k], 1.0, 0.5, 1.0);
    vec3 c = vec3(0.1, 0.2, 0.3);
    c.xy = c.yz * scale;
    float arr[3] = float[3](0.25, 1e-3, 2.0);
    items[k].a = vec4(c, mix(arr[0], arr[2], t));
    items[k].a.w += fract(-1.75) + clamp(p.x, -1.0, 1.0) * 0.0;
    items[k].u = uvec2(total, uint(-3.0));
    items[k].a.x = p.x;
}
@end

@fs probe_fs
in vec2 uv;
flat in float cutoff;
out vec4 out_color;

void main() {
    if (uv.x < cutoff) discard;
    out_color = vec4(uv, exp(0.0), int(2.9));
}
@end
"""

HARNESS = r"""
#include "glsl.h"
#include <cstdio>
#include <ucontext.h>

namespace wg {
ucontext_t sched;
ucontext_t fib[4];
bool done[4];
char stacks[4][65536];
int cur;
void (*entry)();
void tramp() { entry(); done[cur] = true; }
void barrier() { swapcontext(&fib[cur], &sched); }
}

namespace cs {
using namespace glsl;
uvec3 gl_GlobalInvocationID, gl_LocalInvocationID, gl_WorkGroupID;
inline void barrier() { wg::barrier(); }
#include "probe_cs.inc"
}

namespace fs {
using namespace glsl;
vec4 gl_FragCoord;
bool gl_discarded;
#include "probe_fs.inc"
}

int main() {
    static float inputs[4] = {1.0f, 2.0f, 3.5f, -4.0f};
    static cs::Item items[4];
    cs::inputs = inputs;
    cs::items = items;
    cs::count = 3;
    cs::t = 0.25f;
    cs::scale = glsl::vec2(2.0f, 4.0f);
    for (int c = 0; c < 4; ++c)
        for (int r = 0; r < 4; ++r) cs::m.c[c].d[r] = (float)(1 + c * 4 + r) * 0.1f;
    wg::entry = cs::stage_main;
    for (int i = 0; i < 4; ++i) {
        getcontext(&wg::fib[i]);
        wg::fib[i].uc_stack.ss_sp = wg::stacks[i];
        wg::fib[i].uc_stack.ss_size = sizeof(wg::stacks[i]);
        wg::fib[i].uc_link = &wg::sched;
        makecontext(&wg::fib[i], wg::tramp, 0);
    }
    for (bool live = true; live;) {
        live = false;
        for (int i = 0; i < 4; ++i) {
            if (wg::done[i]) continue;
            wg::cur = i;
            cs::gl_LocalInvocationID = glsl::uvec3((uint32_t)i, 0u, 0u);
            cs::gl_GlobalInvocationID = glsl::uvec3((uint32_t)i, 0u, 0u);
            swapcontext(&wg::sched, &wg::fib[i]);
            live = true;
        }
    }
    for (int k = 0; k < 4; ++k)
        std::printf("%a %a %a %a %u %u\n", items[k].a.x, items[k].a.y, items[k].a.z, items[k].a.w, items[k].u.x,
                    items[k].u.y);
    for (float x : {0.2f, 0.7f}) {
        fs::uv = glsl::vec2(x, 0.5f);
        fs::cutoff = 0.5f;
        fs::gl_discarded = false;
        fs::out_color = glsl::vec4(-1.0f);
        fs::stage_main();
        std::printf("%d %a %a %a %a\n", (int)fs::gl_discarded, fs::out_color.x, fs::out_color.y, fs::out_color.z,
                    fs::out_color.w);
    }
    return 0;
}
"""


def _f32(x):
    return np.float32(x)


@pytest.fixture(scope="module")
def probe(tmp_path_factory):
    d = tmp_path_factory.mktemp("glsl_probe")
    src = d / "probe.glsl"
    src.write_text(STAGES)
    for stage in ("probe_cs", "probe_fs"):
        assert extract.main(["extract.py", str(src), stage, str(d / f"{stage}.inc")]) == 0
    (d / "main.cpp").write_text(HARNESS)
    oracle = ROOT / "oracle"
    exe = d / "probe"
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-fopenmp", "-c", str(oracle / "gs_oracle.c"), "-o",
                    str(d / "gs_oracle.o")], check=True)
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-Wall", "-Werror", "-Wno-unused",
                    f"-I{oracle / 'glsl'}", f"-I{d}", str(d / "main.cpp"), str(d / "gs_oracle.o"), "-fopenmp", "-lm",
                    "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    return d, [line.split() for line in out if line]


def test_translation_rules(probe):
    d, _ = probe
    cs = (d / "probe_cs.inc").read_text()
    assert "layout" not in cs and "@" not in cs.split("\n", 1)[1]
    assert "uniform" not in cs and "buffer" not in cs and "shared" not in cs
    assert "Item* items = nullptr;" in cs and "float* inputs = nullptr;" in cs
    assert "mat4 m;" in cs and "uint partial[4];" in cs
    assert "{0.25f, 1e-3f, 2.0f}" in cs           # array constructor + literal suffixes
    assert "u32_of(inputs[lid] * 2.5f)" in cs and "i32_of(gl_GlobalInvocationID.x)" in cs
    assert "void stage_main()" in cs and "void main" not in cs
    fs = (d / "probe_fs.inc").read_text()
    assert "vec2 uv;" in fs and "float cutoff;" in fs and "vec4 out_color;" in fs
    assert "{ gl_discarded = true; return; }" in fs


def test_compute_stage_semantics(probe):
    _, rows = probe
    m = [[_f32(1 + c * 4 + r) * _f32(0.1) for r in range(4)] for c in range(4)]
    inputs = [_f32(1.0), _f32(2.0), _f32(3.5), _f32(-4.0)]
    # shared partial sums after the barrier: uint(x * 2.5) saturating (negative -> 0)
    total = sum(int(max(0.0, float(x * _f32(2.5)))) for x in inputs)
    for k in range(3):
        a = [float.fromhex(v) for v in rows[k][:4]]
        u = [int(v) for v in rows[k][4:]]
        v = [inputs[k], _f32(1.0), _f32(0.5), _f32(1.0)]
        px = ((m[0][0] * v[0] + m[1][0] * v[1]) + m[2][0] * v[2]) + m[3][0] * v[3]   # left to right, no FMA
        assert a[0] == float(px)
        # c.xy = c.yz * scale (the swizzle read happens before the write)
        assert a[1] == float(_f32(0.3) * _f32(4.0)) and a[2] == float(_f32(0.3))
        mix = _f32(0.25) * (_f32(1.0) - _f32(0.25)) + _f32(2.0) * _f32(0.25)
        assert a[3] == float(mix + (_f32(-1.75) - np.floor(_f32(-1.75))))
        assert u == [total, 0]
    assert [float.fromhex(v) for v in rows[3][:4]] == [0.0, 0.0, 0.0, 0.0]   # k >= count returned


def test_fragment_stage_discard(probe):
    _, rows = probe
    kept, disc = rows[5], rows[4]
    assert disc[0] == "1" and float.fromhex(disc[1]) == -1.0
    assert kept[0] == "0"
    assert [float.fromhex(v) for v in kept[1:]] == [float(_f32(0.7)), 0.5, 1.0, 2.0]
