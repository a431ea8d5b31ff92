"""WGSL -> C++ source translator for the reference's compute shaders.

TEST INFRASTRUCTURE ONLY.  The reference (wooningeire/nprush) is TypeScript +
WGSL and there is no WebGPU runtime here, so its shaders cannot be executed as
shipped.  This module rewrites the reference's OWN shader source text
(src/lib/gpu/{splat,bezier}_{backward,step,adc}.wgsl, read from the reference
checkout at build time, never copied into this repository) into C++ that runs
on the host through the fiber runtime in oracle/wgsl_rt.h.  The compiled result
lands in oracle/_ref/ and is the ground truth against which the hand-written
oracle restatement (oracle/nps_oracle.cpp) is pinned.

Placeholders `{@KEY}` are substituted exactly as the reference does in
src/lib/gpu/constants.ts:47-55 (injectWgslConstants), with the values of
GPU_CONSTANTS (constants.ts:5-42) plus the per-manager sizes
(GpuSplatOptimizerManager.ts:127-136, GpuBezierOptimizerManager.ts:146-158).

Only the WGSL subset used by those six shaders is supported; anything else
raises TranslateError so a silent mistranslation cannot happen.
"""
from __future__ import annotations

import re
from dataclasses import dataclass, field

TRANSLATOR_VERSION = "6"


class TranslateError(RuntimeError):
    pass


def js_number(v) -> str:
    """String(v) as JavaScript would print a number (only what we need)."""
    if isinstance(v, bool):
        return "true" if v else "false"
    if isinstance(v, int) or (isinstance(v, float) and v.is_integer() and abs(v) < 1e21):
        return str(int(v))
    r = repr(float(v))
    if "e" in r:
        mant, exp = r.split("e")
        exp_i = int(exp)
        if -7 < exp_i < 21:
            # JavaScript prints these without an exponent
            from decimal import Decimal
            return format(Decimal(r), "f")
        return f"{mant}e{'+' if exp_i > 0 else '-'}{abs(exp_i)}"
    return r


def inject(src: str, subs: dict) -> str:
    def rep(m):
        key = m.group(1)
        if key not in subs:
            raise TranslateError(f"placeholder {{@{key}}} not defined")
        return js_number(subs[key]) if not isinstance(subs[key], str) else subs[key]
    return re.sub(r"\{@([A-Z0-9_]+)\}", rep, src)


# ---------------------------------------------------------------- tokenizer
_TOKEN_RE = re.compile(
    r"""
    (?P<ws>\s+)
  | (?P<lc>//[^\n]*)
  | (?P<bc>/\*.*?\*/)
  | (?P<num>0[xX][0-9a-fA-F]+[iu]?|(?:\d+\.\d*|\.\d+|\d+)(?:[eE][+-]?\d+)?[iufh]?)
  | (?P<id>[A-Za-z_][A-Za-z0-9_]*)
  | (?P<op><<=|>>=|->|<=|>=|==|!=|&&|\|\||\+=|-=|\*=|/=|%=|&=|\|=|\^=|<<|\+\+|--|[-+*/%<>=!&|^~(){}\[\],;:.@])
    """,
    re.S | re.X,
)


@dataclass
class Tok:
    kind: str
    text: str


def tokenize(src: str) -> list[Tok]:
    out = []
    pos = 0
    while pos < len(src):
        m = _TOKEN_RE.match(src, pos)
        if not m:
            raise TranslateError(f"cannot tokenize near: {src[pos:pos+40]!r}")
        pos = m.end()
        kind = m.lastgroup
        if kind in ("ws", "lc", "bc"):
            continue
        out.append(Tok(kind, m.group(kind)))
    return out


SCALARS = {"f32": "f32", "u32": "u32", "i32": "i32", "bool": "bool"}
VECS = {f"vec{n}{s}": f"vec{n}{s}" for n in (2, 3, 4) for s in "fui"}
BUILTINS = {
    "select", "min", "max", "clamp", "abs", "sqrt", "exp", "log", "pow", "sin", "cos",
    "floor", "fract", "step", "smoothstep", "dot", "cross", "length", "countTrailingZeros",
    "atomicAdd", "atomicOr", "atomicExchange", "atomicLoad", "atomicStore",
    "textureLoad", "textureStore", "textureDimensions", "workgroupBarrier", "storageBarrier",
    "textureSampleLevel", "textureSample", "atan2", "asin", "acos", "atan", "tan", "reflect", "normalize", "sign",
}
CXX_KEYWORDS = {
    "new", "delete", "this", "class", "template", "typename", "union", "auto", "register",
    "char", "short", "long", "double", "int", "float", "unsigned", "signed", "static",
    "extern", "inline", "namespace", "operator", "private", "public", "protected", "friend",
    "virtual", "explicit", "mutable", "typeid", "sizeof", "goto", "try", "catch", "throw",
    "and", "or", "not", "xor", "bitand", "bitor", "compl", "default", "case", "do", "export",
    "volatile", "wchar_t", "using", "enum", "asm", "main", "mk", "sw", "vec", "warray",
    "mkarr", "pool", "launch",
}
SWZ = {"x": 0, "y": 1, "z": 2, "w": 3, "r": 0, "g": 1, "b": 2, "a": 3}


@dataclass
class Module:
    structs: list = field(default_factory=list)      # (name, [(fname, ctype)])
    bindings: list = field(default_factory=list)     # (group, binding, name, space, ctype)
    workgroup: list = field(default_factory=list)    # (name, ctype)
    consts: list = field(default_factory=list)       # C++ text
    funcs: list = field(default_factory=list)        # C++ text
    entry: str | None = None
    wgsize: tuple = (1, 1, 1)
    field_names: set = field(default_factory=set)
    fn_names: set = field(default_factory=set)
    stage_fns: list = field(default_factory=list)    # (name, [param types]) of @vertex / @fragment functions


class Translator:
    def __init__(self, toks: list[Tok]):
        self.t = toks
        self.i = 0
        self.m = Module()
        self.binding_names: set[str] = set()

    # -- token helpers
    def peek(self, k=0):
        j = self.i + k
        return self.t[j] if j < len(self.t) else Tok("eof", "")

    def next(self):
        tok = self.peek()
        self.i += 1
        return tok

    def expect(self, text):
        tok = self.next()
        if tok.text != text:
            raise TranslateError(f"expected {text!r}, got {tok.text!r} (token {self.i})")
        return tok

    def attrs(self):
        out = []
        while self.peek().text == "@":
            self.next()
            name = self.next().text
            args = []
            if self.peek().text == "(":
                self.next()
                depth = 1
                cur = []
                while depth:
                    tok = self.next()
                    if tok.text == "(":
                        depth += 1
                    elif tok.text == ")":
                        depth -= 1
                        if depth == 0:
                            break
                    if tok.text == "," and depth == 1:
                        args.append(" ".join(c.text for c in cur))
                        cur = []
                    else:
                        cur.append(tok)
                if cur:
                    args.append(" ".join(c.text for c in cur))
            out.append((name, args))
        return out

    # -- types
    def parse_type(self) -> str:
        tok = self.next()
        name = tok.text
        if name in SCALARS:
            return SCALARS[name]
        if name in VECS:
            return VECS[name]
        if name in ("mat4x4f",):
            return "mat4x4f"
        if name in ("vec2", "vec3", "vec4", "mat4x4"):
            self.expect("<")
            inner = self.parse_type()
            self.close_angle()
            if name == "mat4x4":
                if inner != "f32":
                    raise TranslateError("only mat4x4<f32> supported")
                return "mat4x4f"
            return f"vec{name[-1]}{ {'f32': 'f', 'u32': 'u', 'i32': 'i'}[inner] }"
        if name == "atomic":
            self.expect("<")
            inner = self.parse_type()
            self.close_angle()
            return inner
        if name == "array":
            self.expect("<")
            inner = self.parse_type()
            if self.peek().text == ">":  # runtime-sized: indexes the bound buffer
                self.close_angle()
                return f"rtarray<{inner}>"
            self.expect(",")
            n = self.expr_until_angle()
            return f"warray<{inner}, {n}>"
        if name == "texture_2d":
            self.expect("<")
            self.parse_type()
            self.close_angle()
            return "texture_2d"
        if name == "texture_storage_2d":
            # texture_storage_2d<format, access>: the host side receives the
            # stored float values (before the format's conversion)
            self.expect("<")
            self.next()
            self.expect(",")
            self.next()
            self.close_angle()
            return "texture_storage_2d"
        if name == "sampler":
            return "sampler"
        if name == "ptr":  # ptr<function, T>
            self.expect("<")
            self.next()
            self.expect(",")
            inner = self.parse_type()
            self.close_angle()
            return f"{inner}*"
        if tok.kind == "id":
            return name  # user struct
        raise TranslateError(f"unknown type {name!r}")

    def close_angle(self):
        tok = self.peek()
        if tok.text == ">":
            self.next()
        elif tok.text == ">>":  # not produced by the tokenizer, kept for safety
            tok.text = ">"
        elif tok.text == ">=":
            tok.text = "="
        else:
            raise TranslateError(f"expected '>' got {tok.text!r}")

    def expr_until_angle(self) -> str:
        parts = []
        depth = 0
        while True:
            tok = self.peek()
            if tok.text == ">" and depth == 0:
                self.next()
                break
            if tok.text in ("(", "<"):
                depth += 1
            if tok.text in (")",):
                depth -= 1
            self.next()
            parts.append(self.cxx_literal(tok) if tok.kind == "num" else tok.text)
        return " ".join(parts)

    # -- literals
    @staticmethod
    def cxx_literal(tok: Tok) -> str:
        s = tok.text
        if s.startswith(("0x", "0X")):
            return s[:-1] if s.endswith("i") else s
        if s.endswith("u"):
            return s
        if s.endswith("i"):
            return s[:-1]
        if s.endswith("h"):
            raise TranslateError("f16 literals unsupported")
        if s.endswith("f"):
            body = s[:-1]
            if "." not in body and "e" not in body.lower():
                body += ".0"
            return body + "f"
        if "." in s or "e" in s.lower():
            if s.endswith("."):
                s += "0"
            return s + "f"
        return s

    def ident(self, name: str) -> str:
        if name in CXX_KEYWORDS:
            return name + "_"
        return name

    # -- top level
    def run(self) -> Module:
        while self.peek().kind != "eof":
            at = self.attrs()
            tok = self.peek()
            if tok.text == "struct":
                self.parse_struct()
            elif tok.text == "var":
                self.parse_global_var(at)
            elif tok.text == "const":
                self.parse_const()
            elif tok.text == "fn":
                self.parse_fn(at)
            elif tok.text == ";":
                self.next()
            else:
                raise TranslateError(f"unexpected top-level token {tok.text!r}")
        return self.m

    def parse_struct(self):
        self.expect("struct")
        name = self.next().text
        self.expect("{")
        fields = []
        while self.peek().text != "}":
            self.attrs()
            fname = self.next().text
            self.expect(":")
            ftype = self.parse_type()
            fields.append((self.ident(fname), ftype))
            self.m.field_names.add(fname)
            if self.peek().text == ",":
                self.next()
        self.expect("}")
        if self.peek().text == ";":
            self.next()
        self.m.structs.append((name, fields))

    def parse_global_var(self, at):
        self.expect("var")
        space = ""
        if self.peek().text == "<":
            self.next()
            parts = []
            while self.peek().text != ">":
                parts.append(self.next().text)
            self.next()
            space = "".join(parts)
        name = self.next().text
        self.expect(":")
        ctype = self.parse_type()
        self.expect(";")
        adict = {a[0]: a[1] for a in at}
        if "binding" in adict:
            g = int(adict["group"][0])
            b = int(adict["binding"][0])
            self.m.bindings.append((g, b, name, space, ctype))
            self.binding_names.add(name)
        elif space == "workgroup":
            self.m.workgroup.append((self.ident(name), ctype))
        else:
            raise TranslateError(f"unsupported global var {name} <{space}>")

    def parse_const(self):
        self.expect("const")
        name = self.next().text
        ctype = None
        if self.peek().text == ":":
            self.next()
            ctype = self.parse_type()
        self.expect("=")
        body = self.expr_tokens_until(";")
        self.expect(";")
        simple = all(re.fullmatch(r"[0-9.eExXa-fA-Fu+\-*/() ]+|[A-Z_][A-Z0-9_]*", p) for p in body.split())
        kw = "constexpr" if simple else "static const"
        self.m.consts.append(f"{kw} {ctype or 'auto'} {self.ident(name)} = {body};")

    def parse_fn(self, at):
        self.expect("fn")
        name = self.next().text
        self.m.fn_names.add(name)
        self.expect("(")
        params = []
        while self.peek().text != ")":
            pat = self.attrs()
            pname = self.next().text
            self.expect(":")
            ptype = self.parse_type()
            params.append((pname, ptype, {a[0]: a[1] for a in pat}))
            if self.peek().text == ",":
                self.next()
        self.expect(")")
        ret = "void"
        if self.peek().text == "->":
            self.next()
            self.attrs()
            ret = self.parse_type()
        adict = {a[0]: a[1] for a in at}
        self.cur_ret = ret  # for `discard`
        body = self.block()
        if "compute" in adict:
            ws = [int(re.sub(r"[ui]$", "", x.strip())) for x in adict["workgroup_size"]]
            while len(ws) < 3:
                ws.append(1)
            self.m.wgsize = tuple(ws)
            mapping = {
                "global_invocation_id": "gid__", "workgroup_id": "wid__",
                "local_invocation_id": "lid__", "local_invocation_index": "lidx__",
                "num_workgroups": "nwg__",
            }
            pre = []
            for pname, ptype, pa in params:
                bname = pa["builtin"][0]
                pre.append(f"  const {ptype} {self.ident(pname)} = {mapping[bname]};")
            cname = "entry__" + name
            self.m.entry = cname
            self.m.funcs.append(
                f"static void {cname}(vec3u gid__, vec3u wid__, vec3u lid__, u32 lidx__, vec3u nwg__) {{\n"
                + "\n".join(pre) + "\n  (void)gid__; (void)wid__; (void)lid__; (void)lidx__; (void)nwg__;\n"
                + body + "\n}\n"
            )
        else:
            # plain functions, and @vertex / @fragment stages as plain functions
            # of their (attribute-annotated) inputs
            plist = ", ".join(f"{pt} {self.ident(pn)}" for pn, pt, _ in params)
            self.m.funcs.append(f"static {ret} {self.ident(name)}({plist}) {{\n{body}\n}}\n")
            if "vertex" in adict or "fragment" in adict:
                self.m.stage_fns.append((self.ident(name), [pt for _, pt, _ in params]))

    # -- statements / expressions (token rewriting)
    def expr_tokens_until(self, stop: str) -> str:
        out = []
        depth = 0
        while True:
            tok = self.peek()
            if tok.kind == "eof":
                raise TranslateError("unexpected eof")
            if depth == 0 and tok.text == stop:
                break
            if tok.text in ("(", "[", "{"):
                depth += 1
            if tok.text in (")", "]", "}"):
                depth -= 1
            out.append(self.rewrite_one())
        return " ".join(x for x in out if x)

    def block(self) -> str:
        self.expect("{")
        out = []
        depth = 1
        while True:
            tok = self.peek()
            if tok.text == "{":
                depth += 1
                self.next()
                out.append("{")
                continue
            if tok.text == "}":
                depth -= 1
                self.next()
                if depth == 0:
                    break
                out.append("}")
                continue
            if tok.text in ("let", "var", "const") and self.peek(1).kind == "id":
                out.append(self.decl())
                continue
            if tok.text == "discard":
                # the invocation ends without output; call_<fn> reports it through wg_discarded()
                self.next()
                self.expect(";")
                out.append("{ discard__ = true; return; }" if self.cur_ret == "void"
                           else "{ discard__ = true; return {}; }")
                continue
            if tok.text in ("loop", "switch", "continuing"):
                raise TranslateError(f"unsupported statement {tok.text}")
            out.append(self.rewrite_one())
        return " ".join(x for x in out if x)

    def decl(self) -> str:
        kw = self.next().text
        name = self.ident(self.next().text)
        ctype = None
        if self.peek().text == ":":
            self.next()
            ctype = self.parse_type()
        if self.peek().text == "=":
            self.next()
            expr = self.expr_tokens_until_stmt_end()
            prefix = "const " if kw in ("let", "const") else ""
            return f"{prefix}{ctype or 'auto'} {name} = {expr}"
        if kw != "var" or ctype is None:
            raise TranslateError(f"declaration of {name} without initializer")
        return f"{ctype} {name}{{}}"

    def expr_tokens_until_stmt_end(self) -> str:
        out = []
        depth = 0
        while True:
            tok = self.peek()
            if depth == 0 and tok.text in (";",):
                break
            if tok.text in ("(", "[", "{"):
                depth += 1
            if tok.text in (")", "]", "}"):
                if depth == 0:
                    break
                depth -= 1
            out.append(self.rewrite_one())
        return " ".join(x for x in out if x)

    def rewrite_one(self) -> str:
        tok = self.next()
        if tok.kind == "num":
            return self.cxx_literal(tok)
        if tok.kind == "op":
            # the tokenizer splits '>>' (it cannot tell a shift from two
            # closing template brackets); in an expression it is a shift
            if tok.text == ">" and self.peek().text in (">", ">="):
                return ">" + self.next().text
            if tok.text == "," and self.peek().text == ")":  # trailing comma in a call
                return ""
            if tok.text == ".":
                nxt = self.peek()
                if nxt.kind == "id" and len(nxt.text) >= 2 and nxt.text not in self.m.field_names and (
                    set(nxt.text) <= set("xyzw") or set(nxt.text) <= set("rgba")
                ):
                    self.next()
                    idx = ",".join(str(SWZ[c]) for c in nxt.text)
                    return f".sw__<{idx}>()"
                if nxt.kind == "id":
                    self.next()
                    return "." + self.ident(nxt.text)
            return tok.text
        # identifiers
        name = tok.text
        nxt = self.peek()
        if name == "array" and nxt.text == "<":
            self.next()
            inner = self.parse_type()
            self.expect(",")
            n = self.expr_until_angle()
            if self.peek().text != "(":
                raise TranslateError("array<> type outside constructor/declaration")
            return f"mkarr<{inner}, {n}>"
        if name == "bitcast" and nxt.text == "<":
            self.next()
            inner = self.parse_type()
            self.close_angle()
            return f"wgsl::bitcast<{inner}>"
        if name in ("vec2", "vec3", "vec4") and nxt.text == "<":
            self.i -= 1
            t = self.parse_type()
            return t + "_"
        if nxt.text == "(" and any(name == sn for sn, _ in self.m.structs):
            # struct constructor: aggregate initialisation
            self.next()
            body = self.expr_tokens_until(")")
            self.expect(")")
            return f"{self.ident(name)}{{{body}}}"
        if name in SCALARS and nxt.text == "(":
            return f"wgsl::{name}_"
        if name in VECS and nxt.text == "(":
            return f"wgsl::{name}_"
        if name in BUILTINS and nxt.text == "(" and name not in self.m.fn_names:
            return f"wgsl::{name}"
        if name in self.binding_names:
            return f"(*{name}__b)"
        if name in ("true", "false"):
            return name
        return self.ident(name)


def translate(src: str, subs: dict, origin: str) -> str:
    text = inject(src, subs)
    tr = Translator(tokenize(text))
    m = tr.run()
    if m.entry is None and not m.stage_fns:
        raise TranslateError("no @compute, @vertex or @fragment entry point")
    out = []
    out.append(f"// Generated by oracle/wgsl2cpp.py v{TRANSLATOR_VERSION} from {origin}.")
    out.append("// Build artefact of the test oracle; not part of the product.")
    out.append('#include "wgsl_rt.h"')
    out.append("namespace refmod {")
    out.append("using namespace wgsl;")
    for name, fields in m.structs:
        out.append(f"struct {name} {{")
        for fname, ftype in fields:
            out.append(f"  {ftype} {fname};")
        out.append("};")
    for c in m.consts:
        out.append(c)
    for g, b, name, space, ctype in m.bindings:
        out.append(f"static {ctype}* {name}__b = nullptr;  // @group({g}) @binding({b}) var<{space}>")
    for name, ctype in m.workgroup:
        out.append(f"static {ctype} {name};  // var<workgroup>")
    out.append("static bool discard__ = false;  // set by `discard` in a fragment stage")
    out.append("static void wg_zero__() {")
    for name, ctype in m.workgroup:
        out.append(f"  std::memset((void*)&{name}, 0, sizeof({name}));")
    out.append("}")
    out.extend(m.funcs)
    # @vertex / @fragment stages with one input: call_<name>(in, out) copies
    # the result out; size_<name>(o) gives sizeof(input), sizeof(result)
    # Several inputs (e.g. @builtin(vertex_index), @builtin(instance_index))
    # are packed in order as the members of one struct.
    for fname, ptypes in m.stage_fns:
        if not ptypes:
            continue
        members = " ".join(f"{pt} a{k};" for k, pt in enumerate(ptypes))
        out.append(f"struct in__{fname} {{ {members} }};")
        args = ", ".join(f"in.a{k}" for k in range(len(ptypes)))
        out.append(f'extern "C" void call_{fname}(const void* in_, void* out) {{')
        out.append(f"  const in__{fname}& in = *(const in__{fname}*)in_;")
        out.append("  discard__ = false;")
        out.append(f"  const auto r = {fname}({args});")
        out.append("  std::memcpy(out, &r, sizeof r);")
        out.append("}")
        out.append(f'extern "C" void size_{fname}(unsigned* o) {{')
        decl = ", ".join(f"std::declval<{pt}>()" for pt in ptypes)
        out.append(f"  o[0] = sizeof(in__{fname}); o[1] = sizeof({fname}({decl}));")
        out.append("}")
    out.append("}  // namespace refmod")
    wx, wy, wz = m.wgsize
    out.append('extern "C" {')
    out.append("int wg_discarded() { return refmod::discard__ ? 1 : 0; }")
    out.append("void wg_bind(int group, int binding, void* p) {")
    for g, b, name, space, ctype in m.bindings:
        if ctype not in ("texture_2d", "texture_storage_2d", "sampler"):
            out.append(f"  if (group == {g} && binding == {b}) refmod::{name}__b = (decltype(refmod::{name}__b))p;")
    out.append("}")
    out.append("void wg_bind_storage_tex(int group, int binding, float* rgba, unsigned w, unsigned h) {")
    for g, b, name, space, ctype in m.bindings:
        if ctype == "texture_storage_2d":
            out.append(
                f"  if (group == {g} && binding == {b}) {{ static wgsl::texture_storage_2d t; t.rgba = rgba; t.w = w;"
                f" t.h = h; refmod::{name}__b = &t; }}"
            )
    out.append("}")
    out.append("void wg_bind_tex(int group, int binding, const float* rgba, unsigned w, unsigned h) {")
    for g, b, name, space, ctype in m.bindings:
        if ctype == "texture_2d":
            out.append(
                f"  if (group == {g} && binding == {b}) {{ static wgsl::texture_2d t; t.rgba = rgba; t.w = w; t.h = h;"
                f" refmod::{name}__b = &t; }}"
            )
    out.append("}")
    out.append("void wg_bind_sampler(int group, int binding, int linear, int address_u, int address_v) {")
    for g, b, name, space, ctype in m.bindings:
        if ctype == "sampler":
            out.append(
                f"  if (group == {g} && binding == {b}) {{ static wgsl::sampler s; s.linear = linear;"
                f" s.address_u = address_u; s.address_v = address_v; refmod::{name}__b = &s; }}"
            )
    out.append("}")
    out.append(f"void wg_size(unsigned* o) {{ o[0] = {wx}; o[1] = {wy}; o[2] = {wz}; }}")
    out.append("void wg_run_one(unsigned x, unsigned y, unsigned z, unsigned gx, unsigned gy, unsigned gz) {")
    if m.entry is not None:
        out.append("  refmod::wg_zero__();")
        out.append(
            f"  wgsl::run_workgroup(refmod::{m.entry}, wgsl::mk<wgsl::u32,3>(x, y, z),"
            f" wgsl::mk<wgsl::u32,3>({wx}u, {wy}u, {wz}u), wgsl::mk<wgsl::u32,3>(gx, gy, gz));"
        )
    else:  # a vertex / fragment module: no compute entry point
        out.append("  (void)x; (void)y; (void)z; (void)gx; (void)gy; (void)gz;")
    out.append("}")
    out.append("void wg_dispatch(unsigned gx, unsigned gy, unsigned gz) {")
    out.append("  for (unsigned z = 0; z < gz; ++z) for (unsigned y = 0; y < gy; ++y) for (unsigned x = 0; x < gx; ++x)")
    out.append("    wg_run_one(x, y, z, gx, gy, gz);")
    out.append("}")
    out.append("}")
    return "\n".join(out) + "\n"
