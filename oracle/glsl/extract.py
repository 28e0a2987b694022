"""Cut one stage out of a reference shader file (sokol-shdc input: `@cs`,
`@vs` or `@fs NAME` ... `@end`) and rewrite it, mechanically, as C++ for
oracle/glsl/glsl.h.

TEST INFRASTRUCTURE ONLY: run by oracle/Makefile at build time on the
reference's own shaders/*.glsl; its output goes to oracle/_ref/glsl/ and is
never committed.  Nothing is changed in what the stage computes:

  - `layout(...)` qualifiers and sokol-shdc `@` annotations are dropped;
  - uniform blocks become their members as namespace-scope variables, buffer
    blocks a pointer per unsized array (`T name[];` -> `T* name`), opaque
    uniforms (texture2D, sampler) plain variables;
  - stage inputs and outputs (`in`/`out`, `flat`) become variables the
    harness sets and reads; `shared` variables plain variables (the harness
    runs one workgroup at a time);
  - GLSL array constructors `T[n](a, b, ...)` become brace initialisers;
  - float literals get an `f` suffix (GLSL literals are single precision,
    C++ ones double);
  - `uint(x)` and `int(x)` become the saturating conversions u32_of / i32_of;
  - `discard;` sets gl_discarded and returns; `main` is renamed stage_main.

A second mode cuts one C function out of a reference source file unchanged
(from its signature line to the brace that closes its body), for functions
the harness runs that live in files too entangled to compile whole:

Usage: python extract.py SHADER.glsl STAGE OUT.inc
       python extract.py --function SOURCE.cpp NAME OUT.inc
"""
from __future__ import annotations

import re
import sys

_FLOAT_LIT = re.compile(r"(?<![\w.])((?:\d+\.\d*|\.\d+)(?:[eE][+-]?\d+)?|\d+[eE][+-]?\d+)(?![\w.])")
_LAYOUT = re.compile(r"\blayout\s*\([^)]*\)\s*")
_BLOCK_HEAD = re.compile(r"^\s*(?:(?:readonly|writeonly|coherent|restrict|volatile)\s+)*(uniform|buffer)\s+\w+\s*\{\s*$")
_BLOCK_END = re.compile(r"^\s*\}\s*\w*\s*;\s*$")
_BLOCK_LINE = re.compile(r"^\s*(?:(?:readonly|writeonly|coherent|restrict|volatile)\s+)*(uniform|buffer)\s+\w+\s*"
                         r"\{(.*)\}\s*;\s*$")
_UNSIZED = re.compile(r"^(\s*)(\w+)\s+(\w+)\s*\[\s*\]\s*;\s*$")
_OPAQUE = re.compile(r"^\s*uniform\s+(texture2D|sampler)\s+(\w+)\s*;\s*$")
_IFACE = re.compile(r"^\s*(?:(?:flat|smooth|noperspective)\s+)?(?:in|out)\s+(\w+)\s+(\w+)\s*;\s*$")
_ARRAY_CTOR = re.compile(r"\b\w+\s*\[\s*\d*\s*\]\s*\(")


def stage_source(text: str, stage: str) -> list[str]:
    lines = text.splitlines()
    head = re.compile(r"^@(cs|vs|fs)\s+" + re.escape(stage) + r"\s*$")
    for i, line in enumerate(lines):
        if head.match(line.strip()):
            out = []
            for body in lines[i + 1:]:
                if body.strip() == "@end":
                    return out
                out.append(body)
            raise ValueError(f"stage {stage}: no @end")
    raise ValueError(f"stage {stage} not found")


def _array_ctors(src: str) -> str:
    while True:
        m = _ARRAY_CTOR.search(src)
        if not m:
            return src
        depth, j = 1, m.end()
        while depth:
            c = src[j]
            depth += (c == "(") - (c == ")")
            j += 1
        src = src[:m.start()] + "{" + src[m.end():j - 1] + "}" + src[j:]


def translate(lines: list[str]) -> str:
    out: list[str] = []
    block = None
    for raw in lines:
        if raw.lstrip().startswith("@"):
            continue
        line = _LAYOUT.sub("", raw)
        if re.match(r"^\s*in\s*;\s*$", line):          # the local_size declaration
            continue
        if block is None:
            m = _BLOCK_LINE.match(line)
            if m:   # a block on one line: its members, one per declaration
                for member in filter(None, (x.strip() for x in m.group(2).split(";"))):
                    u = _UNSIZED.match(member + ";")
                    out.append(f"{u.group(2)}* {u.group(3)} = nullptr;" if m.group(1) == "buffer" and u
                               else member + ";")
                continue
            m = _BLOCK_HEAD.match(line)
            if m:
                block = m.group(1)
                continue
        else:
            if _BLOCK_END.match(line):
                block = None
                continue
            if block == "buffer":
                m = _UNSIZED.match(line)
                if m:
                    line = f"{m.group(1)}{m.group(2)}* {m.group(3)} = nullptr;"
            out.append(line)
            continue
        line = re.sub(r"^(\s*)shared\s+", r"\1", line)
        m = _OPAQUE.match(line)
        if m:
            line = f"{m.group(1)} {m.group(2)};"
        m = _IFACE.match(line)
        if m:
            line = f"{m.group(1)} {m.group(2)};"
        out.append(line)
    src = "\n".join(out) + "\n"
    src = _array_ctors(src)
    src = _FLOAT_LIT.sub(lambda m: m.group(1) + "f", src)
    src = re.sub(r"\buint\s*\(", "u32_of(", src)
    src = re.sub(r"\bint\s*\(", "i32_of(", src)
    src = re.sub(r"\bdiscard\s*;", "{ gl_discarded = true; return; }", src)
    src = re.sub(r"\bvoid\s+main\s*\(\s*\)", "void stage_main()", src)
    return src


def c_function(text: str, name: str) -> str:
    m = re.search(r"^[^\n;{}]*\b" + re.escape(name) + r"\s*\([^)]*\)\s*\{", text, re.M)
    if not m:
        raise ValueError(f"function {name} not found")
    depth, j = 1, m.end()
    while depth:
        c = text[j]
        depth += (c == "{") - (c == "}")
        j += 1
    return text[m.start():j] + "\n"


def main(argv: list[str]) -> int:
    if len(argv) == 5 and argv[1] == "--function":
        path, name, dst = argv[2:]
        with open(path, encoding="utf-8") as f:
            body = c_function(f.read(), name)
        with open(dst, "w", encoding="utf-8") as f:
            f.write(f"// Cut by oracle/glsl/extract.py from the reference's {path.split('/')[-1]}, "
                    f"function {name}.  Do not edit.\n")
            f.write(body)
        return 0
    if len(argv) != 4:
        print(__doc__.strip().splitlines()[-2:], file=sys.stderr)
        return 2
    path, stage, dst = argv[1:]
    with open(path, encoding="utf-8") as f:
        text = f.read()
    body = translate(stage_source(text, stage))
    with open(dst, "w", encoding="utf-8") as f:
        f.write(f"// Generated by oracle/glsl/extract.py from the reference's {path.split('/')[-1]}, "
                f"stage {stage}.  Do not edit.\n")
        f.write(body)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
