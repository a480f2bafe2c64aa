#!/usr/bin/env python3
"""Rewrite the cube-tracing GLSL shader sources into C++ that the oracle
compiles on the host.

TEST INFRASTRUCTURE ONLY -- part of the parity oracle.  The product library
never includes what this script writes.

Input : the reference checkout ($CT_REF_DIR, else the path refdir.py finds),
        files under src/shaders/.
Output: oracle/_ref/gen/<same file name>, git-ignored.  Nothing of the
        reference is committed; the rewritten copies only live in the build
        directory next to the compiled oracle library.

Every rewrite is mechanical and keeps the shader's arithmetic and control
flow unchanged:

  1. `#extension` lines are dropped.
  2. `layout(buffer_reference, scalar) buffer NAME {T f[]; };` becomes
     `GLSL_BUFREF_ARRAY(NAME, T, f)` (or `GLSL_BUFREF_ONE` without `[]`);
     every other `layout(...)` line (payload / push-constant / workgroup
     declarations) is dropped -- the harness declares those objects itself.
  3. Parameter qualifiers: `inout T x` / `out T x` become `T &x`,
     `const in` becomes `const`, a bare `in` is dropped.
  4. Floating literals without a suffix get `f` (GLSL literals are single
     precision, C++ ones are double).
  5. Scalar constructor casts (`uint(x)`, `daxa_u32(x)`, `int(x)`, `float(x)`
     and the daxa spellings) call the shim's glsl_u32/glsl_i32/glsl_f32,
     which implement GLSL's conversion rules (saturating float->uint).
  6. `T v = ... v ...;` (a name used inside its own initialiser, which GLSL
     resolves to the outer object because a variable's scope starts after
     its initialiser) becomes `T v = ... ::v ...;`, and every `case` of a
     switch gets its own block so that C++ accepts jumps over declarations
     made in an earlier case (GLSL shares one scope across the cases).
  7. Vector, matrix and struct constructor calls `T(a, b)` become `T{a, b}`.
     C++ sequences brace-initialiser arguments left to right, which is the
     GLSL argument evaluation order; this matters where several arguments
     draw from the same random sequence, e.g. `vec2(rnd(seed), rnd(seed))`.
  8. Read-only swizzles `.xyz .xy .yz .zx` (and the `.VW` macro parameter in
     Box.glsl's TEST macro) become member-function calls.
  9. `#define VOXEL_EXTENT 0.03125f` is replaced by the build-time value
     CT_VOXEL_EXTENT, since the scene scale is a parameter of the workload.
 11. The hybrid shift switch: generate_path's `path.use_hybrid_shift = false`
     (path_state.glsl:237) becomes `params.shift_mapping ==
     SHIFT_MAPPING_HYBRID`, and the shift mapping rgen.glsl passes in its
     scene parameters (SHIFT_MAPPING_RECONNECTION, rgen.glsl:282, 437) the
     variable ct_pt_shift_mapping (the reference's value by default).  The
     reference's compute_shifted_integrand_hybrid (shift.glsl:352-444) is
     left as a declaration: its random-replay data is stubbed
     (path_reservoir.glsl:37-58), its producer commented out
     (indirect_illumination.glsl:300-302), and as written it returns a zero
     Jacobian, so the oracle defines the function itself (oracle_main.cpp).
     With the default shift mapping none of this is reached.
 10. The reuse constants that the CUDA path takes as run-time parameters
     (ct_params: RIS candidate counts, temporal caps, the spatial neighbour
     count and radius, MAX_DISTANCE_TO_HIT, the PT neighbour count and
     radius, include/defines.glsl:34-62) lose their `const` and become
     static namespace-scope variables that keep the reference value as their
     initial value; TAA's `#define ALPHA 0.8` (compute/taa.glsl:13) names the
     variable ct_taa_alpha.  oracle_set_params (oracle_main.cpp) sets them
     per run.  The one array bound among them, `[MAX_NUM_OF_NEIGHBORS]`
     (restir_resampling.glsl:429), becomes the fixed capacity
     CT_ORACLE_MAX_NEIGHBORS.

With --fp64 the output goes to oracle/_ref/gen64 for the double-precision
build of the same code: rule 4 is left out (literals stay double) and the
GLSL type name `float` becomes the shim's ct_real (double in that build).
"""
import os
import re
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from refdir import reference_dir  # noqa: E402

REF = reference_dir()
SHADERS = os.path.join(REF, "src", "shaders")
HERE = os.path.dirname(os.path.abspath(__file__))
FP64 = "--fp64" in sys.argv[1:]
OUT = os.path.join(HERE, "_ref", "gen64" if FP64 else "gen")

FILES = [
    "shared.inl",
    "include/defines.glsl",
    "glsl/random.glsl",
    "glsl/prng.glsl",
    "glsl/Box.glsl",
    "glsl/primitives.glsl",
    "glsl/mat.glsl",
    "glsl/light.glsl",
    "glsl/bounce.glsl",
    "glsl/direct_light_info.glsl",
    "glsl/motion_vectors.glsl",
    "glsl/restir_di/reservoir.glsl",
    "glsl/restir_di/pairwise_mis.glsl",
    "glsl/restir_di/restir_resampling.glsl",
    "glsl/restir_pt/path_reservoir.glsl",
    "glsl/restir_pt/path_builder.glsl",
    "glsl/restir_pt/path_state.glsl",
    "glsl/restir_pt/path_tracer.glsl",
    "glsl/restir_pt/shift.glsl",
    "glsl/restir_pt/indirect_illumination.glsl",
    "glsl/raytracing/rgen.glsl",
    "glsl/raytracing/rchit.glsl",
    "glsl/raytracing/rmiss.glsl",
    "glsl/raytracing/rint.glsl",
    "glsl/raytracing/rcall_scatter.glsl",
    "glsl/compute/taa.glsl",
]

VEC_TYPES = [
    "daxa_f32vec2", "daxa_f32vec3", "daxa_f32vec4", "daxa_i32vec2", "daxa_i32vec3",
    "daxa_u32vec2", "daxa_u32vec3", "daxa_f32mat4x4", "daxa_f32mat3x3",
    "vec2", "vec3", "vec4", "ivec2", "ivec3", "uvec2", "uvec3", "bvec2", "bvec3", "bvec4",
    "mat3", "mat4",
]


def strip_comments(src):
    """Remove // and /* */ comments, keeping line structure."""
    out = []
    i, n = 0, len(src)
    while i < n:
        if src.startswith("//", i):
            j = src.find("\n", i)
            if j < 0:
                j = n
            i = j
        elif src.startswith("/*", i):
            j = src.find("*/", i + 2)
            j = n if j < 0 else j + 2
            out.append(" ")
            i = j
        else:
            out.append(src[i])
            i += 1
    return "".join(out)


def braces_for_ctors(src, names):
    pat = re.compile(r"\b(" + "|".join(sorted(names, key=len, reverse=True)) + r")\s*\(")
    s = list(src)
    text = src
    pos = 0
    while True:
        m = pat.search(text, pos)
        if not m:
            break
        # skip declarations such as `struct Ray (`, never present, and
        # function definitions whose return type is the struct name followed
        # by a name are not matched because the name is not followed by '('.
        open_i = m.end() - 1
        depth = 0
        j = open_i
        while j < len(text):
            c = text[j]
            if c == "(":
                depth += 1
            elif c == ")":
                depth -= 1
                if depth == 0:
                    break
            j += 1
        if j >= len(text):
            raise RuntimeError("unbalanced constructor call near: " + text[m.start():m.start() + 80])
        s[open_i] = "{"
        s[j] = "}"
        text = "".join(s)
        pos = m.end()
    return text


KEYWORDS = {"return", "else", "case", "default", "typedef", "goto", "break", "continue", "do", "if", "while", "for", "switch"}


def qualify_self_init(src):
    """`T v = ... v ...;` -> `T v = ... ::v ...;`.

    In GLSL a variable's scope begins after its initialiser, so a name used
    inside its own initialiser denotes the outer (global) object; in C++ it
    would denote the variable being declared."""
    pat = re.compile(r"(^|[;{}]\s*)((?:const\s+)?(\w+)\s+)(\w+)(\s*=(?!=))([^;]*;)", re.M)

    def repl(m):
        if m.group(3) in KEYWORDS:
            return m.group(0)
        name = m.group(4)
        init = re.sub(r"(?<![\w.:])" + re.escape(name) + r"\b", "::" + name, m.group(6))
        return m.group(1) + m.group(2) + name + m.group(5) + init

    return pat.sub(repl, src)


def scope_switch_cases(src):
    """Give every case of a switch its own block: `case A: stmts` ->
    `case A: { stmts }`.  GLSL lets a case jump over declarations made by an
    earlier case (they share the switch scope); C++ rejects that.  Braces do
    not change fall-through, so control flow is unchanged."""
    out = []
    i = 0
    n = len(src)
    sw = re.compile(r"\bswitch\s*\(")
    while True:
        m = sw.search(src, i)
        if not m:
            out.append(src[i:])
            break
        # find the switch body's opening brace
        j = m.end()
        depth = 1
        while depth:
            depth += {"(": 1, ")": -1}.get(src[j], 0)
            j += 1
        k = src.index("{", j)
        out.append(src[i:k + 1])
        # walk the body at depth 1, wrapping case sections
        depth = 1
        pos = k + 1
        open_case = False
        body_start = pos
        while depth:
            c = src[pos]
            if c == "{":
                depth += 1
            elif c == "}":
                depth -= 1
                if depth == 0:
                    break
            if depth == 1:
                lm = re.match(r"(case\b[^:]*|default\s*):", src[pos:])
                if lm and (pos == 0 or not (src[pos - 1].isalnum() or src[pos - 1] == "_")):
                    out.append(scope_switch_cases(src[body_start:pos]))
                    if open_case:
                        out.append("} ")
                    out.append(lm.group(0) + " {")
                    open_case = True
                    pos += lm.end()
                    body_start = pos
                    continue
            pos += 1
        out.append(scope_switch_cases(src[body_start:pos]))
        if open_case:
            out.append("} ")
        out.append("}")
        i = pos + 1
    return "".join(out)


# rule 10: reference constants the oracle takes as run-time parameters
RUNTIME_CONSTANTS = [
    "MIN_RIS_POINT_SAMPLE_COUNT", "MAX_RIS_POINT_SAMPLE_COUNT", "MIN_RIS_ENV_SAMPLE_COUNT",
    "MAX_RIS_ENV_SAMPLE_COUNT", "MIN_RIS_CUBE_SAMPLE_COUNT", "MAX_RIS_CUBE_SAMPLE_COUNT",
    "MIN_INFLUENCE_FROM_THE_PAST_THRESHOLD", "MAX_INFLUENCE_FROM_THE_PAST_THRESHOLD",
    "MIN_NUM_OF_NEIGHBORS", "MAX_NUM_OF_NEIGHBORS", "MIN_NEIGHBORS_RADIUS", "MAX_NEIGHBORS_RADIUS",
    "MAX_DISTANCE_TO_HIT", "MAX_INFLUENCE_FROM_THE_PAST_THRESHOLD_PT", "NEIGHBOR_COUNT", "NEIGHBOR_RADIUS",
    "NEAR_FIELD_DISTANCE",
]


def declaration_only(src, signature_start):
    """Rule 11: the function whose definition starts with `signature_start`
    keeps only its declaration."""
    i = src.find(signature_start)
    if i < 0:
        raise RuntimeError(f"not found: {signature_start}")
    j = src.index("(", i)
    depth = 0
    while True:
        c = src[j]
        depth += {"(": 1, ")": -1}.get(c, 0)
        j += 1
        if depth == 0:
            break
    k = src.index("{", j)
    depth = 0
    m = k
    while True:
        c = src[m]
        depth += {"{": 1, "}": -1}.get(c, 0)
        m += 1
        if depth == 0:
            break
    return src[:j] + ";" + src[m:]


def hybrid_switch(src):
    """Rule 11 (see the module docstring)."""
    if "void generate_path(" in src:
        g = src.index("void generate_path(")
        k = src.index("path.use_hybrid_shift = false;", g)
        src = src[:k] + "path.use_hybrid_shift = params.shift_mapping == SHIFT_MAPPING_HYBRID;" + \
            src[k + len("path.use_hybrid_shift = false;"):]
    if "SCENE_PARAMS params = SCENE_PARAMS(" in src:
        src = re.sub(r"(SCENE_PARAMS params = SCENE_PARAMS\([^;]*?)SHIFT_MAPPING_RECONNECTION", r"\1ct_pt_shift_mapping",
                     src, flags=re.S)
    if "daxa_f32vec3 compute_shifted_integrand_hybrid(" in src:
        src = declaration_only(src, "daxa_f32vec3 compute_shifted_integrand_hybrid(")
    return src


def runtime_constants(src):
    """Rule 10 (see the module docstring)."""
    for name in RUNTIME_CONSTANTS:
        # internal linkage: the FP32 and FP64 builds are loaded into one
        # process, and `inline` variables would be bound to one definition
        src, n = re.subn(r"(?m)^(\s*)const\s+(\w+)\s+" + name + r"\s*=", r"\1static \2 " + name + " =", src)
        if n > 1:
            raise RuntimeError(f"{name} declared {n} times")
    src = re.sub(r"\[\s*MAX_NUM_OF_NEIGHBORS\s*\]", "[CT_ORACLE_MAX_NEIGHBORS]", src)
    src = re.sub(r"(?m)^\s*#define\s+ALPHA\s+0\.8f?\s*$", "#define ALPHA ct_taa_alpha", src)
    return src


def transform(src, struct_names):
    src = strip_comments(src)
    lines = []
    for line in src.split("\n"):
        st = line.strip()
        if st.startswith("#extension"):
            lines.append("")
            continue
        m = re.match(r"\s*layout\(buffer_reference,\s*scalar\)\s*buffer\s+(\w+)\s*\{\s*(\w+)\s+(\w+)\s*(\[\])?\s*;\s*\}\s*;", line)
        if m:
            macro = "GLSL_BUFREF_ARRAY" if m.group(4) else "GLSL_BUFREF_ONE"
            lines.append(f"{macro}({m.group(1)}, {m.group(2)}, {m.group(3)})")
            continue
        if st.startswith("layout("):
            lines.append("")
            continue
        if re.match(r"\s*#define\s+VOXEL_EXTENT\s+0\.03125f", line):
            lines.append("#define VOXEL_EXTENT CT_VOXEL_EXTENT")
            continue
        lines.append(line)
    src = "\n".join(lines)

    # 10. run-time reuse parameters
    src = runtime_constants(src)

    # 11. the hybrid shift switch
    src = hybrid_switch(src)

    # 3. parameter qualifiers
    src = re.sub(r"\bconst\s+in\s+", "const ", src)
    src = re.sub(r"\b(inout|out)\s+((?:const\s+)?\w+)\s+(\w+)", r"\2 &\3", src)
    src = re.sub(r"([(,]\s*)in\s+(?=\w+\s+\w+\s*[,)\[])", r"\1", src)

    # 4. float literals -> single precision
    if not FP64:
        src = re.sub(r"(?<![\w.])((?:\d+\.\d*|\.\d+)(?:[eE][+-]?\d+)?|\d+[eE][+-]?\d+)(?![\w.])", r"\1f", src)

    # 5. scalar constructor casts
    src = re.sub(r"\b(?:daxa_u32|uint)\s*\(", "glsl_u32(", src)
    src = re.sub(r"\b(?:daxa_i32|int)\s*\(", "glsl_i32(", src)
    src = re.sub(r"\b(?:daxa_f32|float)\s*\(", "glsl_f32(", src)
    if FP64:
        src = re.sub(r"\bfloat\b", "ct_real", src)

    # 6. names used inside their own initialiser denote the outer object
    src = qualify_self_init(src)

    # 6b. each switch case gets its own scope
    src = scope_switch_cases(src)

    # 7. constructor calls -> brace initialisation (left-to-right evaluation)
    src = braces_for_ctors(src, VEC_TYPES + sorted(struct_names))

    # 8. swizzles
    src = re.sub(r"\.(xyz|xy|yz|zx|VW)\b(?!\s*\()", r".\1()", src)
    return src


def main():
    if not os.path.isdir(SHADERS):
        print(f"reference shaders not found under {SHADERS}", file=sys.stderr)
        return 2
    os.makedirs(OUT, exist_ok=True)
    raw = {}
    for rel in FILES:
        with open(os.path.join(SHADERS, rel)) as f:
            raw[rel] = f.read()
    structs = set()
    for txt in raw.values():
        structs.update(re.findall(r"\bstruct\s+(\w+)\s*\{", strip_comments(txt)))
    structs.discard("LCG")
    found = {n for t in raw.values() for n in RUNTIME_CONSTANTS if re.search(r"\bconst\s+\w+\s+" + n + r"\s*=", t)}
    if found != set(RUNTIME_CONSTANTS) or not re.search(r"#define\s+ALPHA\s+0\.8", raw["glsl/compute/taa.glsl"]):
        print(f"reference constants not found: {sorted(set(RUNTIME_CONSTANTS) - found)}", file=sys.stderr)
        return 2
    for rel, txt in raw.items():
        out = transform(txt, structs)
        with open(os.path.join(OUT, os.path.basename(rel)), "w") as f:
            f.write(f"// generated from src/shaders/{rel} by oracle/transform.py; do not edit\n")
            f.write(out)
    print(f"wrote {len(FILES)} files to {OUT}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
