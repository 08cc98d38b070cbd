"""Mechanical translation of the reference's WGSL compute shaders into C++.

TEST INFRASTRUCTURE ONLY.  The reference's hot path is WGSL run by wgpu on a
Vulkan ray-query device; neither exists on this machine.  This script turns
the shader source, where it lies in the reference tree, into C++ that
oracle/ref_harness.cpp runs on the CPU, so that the oracle's hand
restatement (oracle/oracle.cpp) can be checked against the reference's own
code.  The output goes to oracle/_ref/ only (git-ignored, never committed).

It handles the subset of WGSL the three shaders use (shader.wgsl,
photon_emit.wgsl, build_grid.wgsl): structs, module-scope const / override /
var declarations, functions, let / var / const statements, if / for / loop /
while, swizzles, and the built-in functions of oracle/ref_runtime.h.  Anything
outside that subset (switch, continuing, a float remainder of two scalars)
stops the translation with an error instead of guessing.

Mapping (the WGSL is never edited by hand):
  fn f(a: T) -> R { ... }   ->  R f(T a) { ... }    (prototypes emitted first)
  let x = e;  var x = e;    ->  const auto x = e;  auto x = e;
  var x: T;                 ->  T x{};              (WGSL zero-initialises)
  if c { ... }              ->  if (c) { ... }
  1.0, 1e-9                 ->  1.0f, 1e-9f         (abstract floats become f32)
  v.xyz, v.rgb, v.r         ->  v.sw<0,1,2>(), v.sw<0,1,2>(), v.x
  max(...), textureStore(...) -> wb_max(...), wb_textureStore(...)
  var<private> x: T         ->  thread_local T x{}  (one value per invocation)
  var<storage> x: array<T>  ->  StorageArray<T> x   (bound by the harness)
  fn main(...)              ->  void cs_main(...)

Usage: python oracle/wgsl_translate.py IN.wgsl OUT.inc NAMESPACE
"""
from __future__ import annotations

import re
import sys

TOKEN_RE = re.compile(
    r"""
    (?P<ws>[ \t\r\f\v]+)
  | (?P<nl>\n)
  | (?P<comment>//[^\n]*|/\*.*?\*/)
  | (?P<num>0[xX][0-9a-fA-F]+[iu]?
          | (?:\d+\.\d*|\.\d+)(?:[eE][+-]?\d+)?[fh]?
          | \d+[eE][+-]?\d+[fh]?
          | \d+[iuf]?)
  | (?P<id>[A-Za-z_][A-Za-z0-9_]*)
  | (?P<op><<=|>>=|->|&&|\|\||==|!=|<=|>=|<<|>>|\+\+|--|\+=|-=|\*=|/=|%=|&=|\|=|\^=|[-+*/%&|^!~<>=(){}\[\];:,.@])
    """,
    re.VERBOSE | re.DOTALL,
)

BUILTINS = {
    "abs", "max", "min", "clamp", "sign", "sqrt", "exp", "cos", "sin", "tan", "atan", "floor", "pow", "dot",
    "length", "normalize", "cross", "reflect", "refract", "select", "arrayLength", "atomicAdd", "atomicLoad",
    "atomicExchange", "textureDimensions", "textureStore", "rayQueryInitialize", "rayQueryProceed",
    "rayQueryGetCommittedIntersection",
}
UNSUPPORTED = {"switch", "continuing", "discard", "bitcast", "workgroupBarrier", "storageBarrier", "textureLoad"}
CPP_KEYWORDS = {
    "auto", "break", "case", "char", "class", "const", "continue", "default", "delete", "do", "double", "else",
    "enum", "extern", "float", "for", "goto", "if", "int", "long", "new", "operator", "private", "protected",
    "public", "register", "return", "short", "signed", "sizeof", "static", "struct", "template", "this", "throw",
    "try", "typedef", "union", "unsigned", "void", "volatile", "while", "namespace", "using", "virtual",
    "friend", "inline", "mutable", "explicit", "export", "typename", "and", "or", "not", "xor",
}
SCALARS = {"f32": "float", "u32": "uint32_t", "i32": "int32_t", "bool": "bool"}
VEC_SHORT = {f"vec{n}{s}": f"vec{n}{s}" for n in (2, 3, 4) for s in "fui"}
SWZ_XYZW = re.compile(r"^[xyzw]{1,4}$")
SWZ_RGBA = re.compile(r"^[rgba]{1,4}$")


class WgslError(RuntimeError):
    pass


def tokenize(src: str) -> list[tuple[str, str, int]]:
    toks, pos, line = [], 0, 1
    while pos < len(src):
        m = TOKEN_RE.match(src, pos)
        if not m:
            raise WgslError(f"line {line}: cannot tokenize {src[pos:pos + 20]!r}")
        kind = m.lastgroup
        text = m.group(kind)
        if kind == "nl":
            toks.append(("nl", "\n", line))
            line += 1
        elif kind == "comment":
            line += text.count("\n")
        elif kind != "ws":
            if kind == "op" and text == ">>":  # split for generics; rejoined in expressions
                toks.append(("op", ">", line))
                toks.append(("op", ">", line))
                toks[-1] = ("op2", ">", line)  # marks the second half of a '>>'
            else:
                toks.append((kind, text, line))
        pos = m.end()
    return toks


class Translator:
    def __init__(self, src: str, ns: str):
        self.t = [tk for tk in tokenize(src)]
        self.ns = ns
        self.i = 0
        ids = [v for k, v, _ in self.t if k != "nl"]
        self.struct_names = {ids[j + 1] for j, v in enumerate(ids[:-1]) if v == "struct"} | {"RayDesc"}
        self.impure = self.impure_functions()
        self.check_evaluation_order()
        self.brace_stack: list[bool] = []
        self.structs: list[str] = []
        self.globals: list[str] = []
        self.protos: list[str] = []
        self.bodies: list[str] = []

    # ---------------------------------------------------------------- token helpers
    def skip_nl(self):
        while self.i < len(self.t) and self.t[self.i][0] == "nl":
            self.i += 1

    def peek(self, k=0) -> str:
        j, seen = self.i, -1
        while j < len(self.t):
            if self.t[j][0] != "nl":
                seen += 1
                if seen == k:
                    return self.t[j][1]
            j += 1
        return ""

    def next(self) -> str:
        self.skip_nl()
        if self.i >= len(self.t):
            raise WgslError("unexpected end of input")
        v = self.t[self.i][1]
        self.i += 1
        return v

    def expect(self, v: str):
        got = self.next()
        if got != v:
            raise WgslError(f"line {self.line()}: expected {v!r}, got {got!r}")

    def line(self) -> int:
        return self.t[min(self.i, len(self.t) - 1)][2]

    # ---------------------------------------------------------------- types
    def parse_type(self) -> str:
        name = self.next()
        if name in SCALARS:
            return SCALARS[name]
        if name in VEC_SHORT:
            return VEC_SHORT[name]
        if name in ("mat3x3f", "mat4x4f", "mat4x3f"):
            return name
        if name in ("ray_query", "acceleration_structure"):
            return name
        if self.peek() != "<":
            return self.ident(name)  # a struct
        self.expect("<")
        args = [self.parse_type_arg()]
        while self.peek() == ",":
            self.next()
            args.append(self.parse_type_arg())
        self.expect(">")
        if re.fullmatch(r"vec[234]", name):
            return f"wgsl_rt::vec<{args[0]}, {name[3]}>"
        if re.fullmatch(r"mat[234]x[234]", name):
            return f"wgsl_rt::mat<{name[3]}, {name[5]}>"
        if name == "array":
            return f"wgsl_rt::warr<{args[0]}, {args[1]}>" if len(args) == 2 else f"wgsl_rt::StorageArray<{args[0]}>"
        if name == "atomic":
            return f"wgsl_rt::Atomic<{args[0]}>"
        if name == "ptr":
            return f"{args[1]}*"
        if name == "texture_storage_2d":
            return "wgsl_rt::texture_storage_2d"
        raise WgslError(f"line {self.line()}: unsupported type {name}<...>")

    def parse_type_arg(self) -> str:
        p = self.peek()
        if re.fullmatch(r"\d+u?", p):
            return self.next().rstrip("u")
        if p in ("function", "private", "storage", "uniform", "workgroup", "read", "write", "read_write",
                 "rgba8unorm"):
            return self.next()
        return self.parse_type()

    @staticmethod
    def ident(name: str) -> str:
        if name == "main":
            return "cs_main"
        return name + "_" if name in CPP_KEYWORDS else name

    # ---------------------------------------------------------------- attributes
    def skip_attributes(self) -> list[str]:
        names = []
        while self.peek() == "@":
            self.next()
            names.append(self.next())
            if self.peek() == "(":
                depth = 0
                while True:
                    v = self.next()
                    depth += v == "("
                    depth -= v == ")"
                    if depth == 0:
                        break
        return names

    # ---------------------------------------------------------------- expressions
    def expr_until(self, stops: set[str], allow_brace=False) -> str:
        """Translate tokens up to (not including) the first stop token at depth 0."""
        out, depth = [], 0
        while True:
            self.skip_nl()
            if self.i >= len(self.t):
                raise WgslError("unexpected end of input in an expression")
            kind, v, _ = self.t[self.i]
            if depth == 0 and v in stops:
                return " ".join(out)
            if v in ("(", "["):
                depth += 1
            elif v in (")", "]"):
                depth -= 1
            elif v == "{" and not allow_brace:
                raise WgslError(f"line {self.line()}: unexpected '{{' in an expression")
            out.append(self.expr_token())
            if self.i < len(self.t) and self.t[self.i][1] == "(" and self.is_constructor(out[-1]):
                # T(...) -> T{...}: a braced list evaluates its elements left to
                # right, as WGSL evaluates arguments; a call's order is unspecified
                self.i += 1
                depth += 1
                out.append("{")
                self.brace_stack.append(True)
            elif v == "(":
                self.brace_stack.append(False)
            elif v == ")":
                if self.brace_stack.pop():
                    out[-1] = "}"

    def expr_token(self) -> str:
        kind, v, line = self.t[self.i]
        self.i += 1
        if kind == "op2":
            return ">"
        if kind == "op" and v == ">" and self.i < len(self.t) and self.t[self.i][0] == "op2":
            self.i += 1
            return ">>"
        if kind == "num":
            return self.number(v)
        if kind == "id":
            if v in UNSUPPORTED:
                raise WgslError(f"line {line}: unsupported construct {v!r}")
            prev = self.t[self.i - 2][1] if self.i >= 2 else ""
            if prev == ".":
                return self.member(v)
            if v in BUILTINS and self.peek() == "(":
                return "wgsl_rt::wb_" + v
            if re.fullmatch(r"vec[234]|mat[234]x[234]|array", v) and self.peek() == "<":
                self.i -= 1
                return self.parse_type()
            if v in SCALARS and self.peek() == "(":
                return {"f32": "wgsl_rt::f32", "u32": "wgsl_rt::u32", "i32": "wgsl_rt::i32", "bool": "bool"}[v]
            if v in VEC_SHORT or v in ("mat3x3f", "mat4x4f", "mat4x3f"):
                return "wgsl_rt::" + v
            if v in ("let", "var", "const", "fn", "struct", "override"):
                raise WgslError(f"line {line}: declaration keyword {v!r} inside an expression")
            return self.ident(v)
        return v

    def is_constructor(self, emitted: str) -> bool:
        name = emitted.split("::")[-1]
        return (name in self.struct_names or re.fullmatch(r"vec[234][fui]|mat[234]x[234]f", name) is not None
                or emitted.startswith("wgsl_rt::vec<") or emitted.startswith("wgsl_rt::mat<")
                or emitted.startswith("wgsl_rt::warr<"))

    # ---------------------------------------------------------------- evaluation order
    def impure_functions(self) -> set[str]:
        """Functions that write module-scope private state or atomics, directly
        or through a call (rand and everything that draws from it)."""
        toks = [v for k, v, _ in self.t if k != "nl"]
        private = {toks[j + 4] for j in range(len(toks) - 4)
                   if toks[j] == "var" and toks[j + 1] == "<" and toks[j + 2] == "private"}
        bodies: dict[str, list[str]] = {}
        j = 0
        while j < len(toks):
            if toks[j] == "fn":
                name = toks[j + 1]
                k = toks.index("{", j)
                depth, e = 0, k
                while True:
                    depth += toks[e] == "{"
                    depth -= toks[e] == "}"
                    if depth == 0:
                        break
                    e += 1
                bodies[name] = toks[k:e + 1]
                j = e
            j += 1
        impure = {n for n, b in bodies.items()
                  if any(b[q] in private and b[q + 1] in ("=", "+=", "-=", "*=", "/=") for q in range(len(b) - 1))
                  or any(a in b for a in ("atomicAdd", "atomicExchange", "textureStore"))}
        changed = True
        while changed:
            changed = False
            for n, b in bodies.items():
                if n not in impure and any(b[q] in impure and b[q + 1] == "(" for q in range(len(b) - 1)):
                    impure.add(n)
                    changed = True
        return impure

    def check_evaluation_order(self):
        """C++ leaves the order of a call's arguments and of most operands
        unspecified; WGSL fixes it left to right.  Braced constructors keep it,
        so a statement may draw from impure functions more than once only as
        distinct arguments of one constructor; anything else is refused."""
        toks = [(v, ln) for k, v, ln in self.t if k != "nl"]
        impure_set = self.impure_functions() if not hasattr(self, "impure") else self.impure
        start = 0
        for j, (v, _) in enumerate(toks):
            if v not in (";", "{", "}"):
                continue
            stmt = toks[start:j]
            start = j + 1
            calls = [q for q in range(len(stmt) - 1) if stmt[q][0] in impure_set and stmt[q + 1][0] == "("]
            if len(calls) < 2:
                continue
            ok = False
            for q in range(len(stmt) - 1):  # a constructor whose distinct arguments hold every call
                name = stmt[q][0]
                if stmt[q + 1][0] != "(" or not (name in self.struct_names or re.fullmatch(r"vec[234][fui]", name)):
                    continue
                depth, arg, owner = 0, 0, {}
                for r in range(q + 1, len(stmt)):
                    t = stmt[r][0]
                    if t in ("(", "["):
                        depth += 1
                    elif t in (")", "]"):
                        depth -= 1
                        if depth == 0:
                            break
                    elif t == "," and depth == 1:
                        arg += 1
                    if r in calls:
                        owner[r] = arg
                if set(owner) == set(calls) and len(set(owner.values())) == len(calls):
                    ok = True
                    break
            if not ok:
                raise WgslError(f"line {stmt[calls[0]][1]}: more than one call to a function with side effects "
                                f"({', '.join(stmt[c][0] for c in calls)}) whose order C++ would not keep")

    @staticmethod
    def number(v: str) -> str:
        if v.lower().startswith("0x"):
            return v[:-1] if v.endswith("i") else v
        if v.endswith("h"):
            raise WgslError("f16 literals are not supported")
        if v.endswith("u"):
            return v
        if v.endswith("i"):
            return v[:-1]
        if v.endswith("f"):
            body = v[:-1]
            return body + ("f" if ("." in body or "e" in body.lower()) else ".0f")
        if "." in v or "e" in v.lower():
            return v + "f"
        return v  # abstract integer

    @staticmethod
    def member(v: str) -> str:
        if SWZ_RGBA.match(v):
            v = v.translate(str.maketrans("rgba", "xyzw"))
        if SWZ_XYZW.match(v):
            if len(v) == 1:
                return v
            return "sw<" + ",".join(str("xyzw".index(c)) for c in v) + ">()"
        return v

    # ---------------------------------------------------------------- statements
    def block(self, indent: str) -> str:
        """Translate a { ... } block (the opening brace is the next token)."""
        self.expect("{")
        lines = ["{"]
        while True:
            self.skip_nl()
            if self.peek() == "}":
                self.next()
                lines.append(indent + "}")
                return "\n".join(lines)
            lines.append(indent + "    " + self.statement(indent + "    "))

    def decl(self, kw: str, terminator: str) -> str:
        name = self.ident(self.next())
        ty = None
        if self.peek() == ":":
            self.next()
            ty = self.parse_type()
        init = None
        if self.peek() == "=":
            self.next()
            init = self.expr_until({terminator})
        if kw == "var":
            if init is None:
                if ty is None:
                    raise WgslError(f"line {self.line()}: var without type or initialiser")
                return f"{ty} {name}{{}}"
            return f"{ty or 'auto'} {name} = {init}"
        if init is None:
            raise WgslError(f"line {self.line()}: {kw} without initialiser")
        return f"const {ty or 'auto'} {name} = {init}"

    def statement(self, indent: str) -> str:
        self.skip_nl()
        v = self.peek()
        if v in ("let", "var", "const"):
            self.next()
            s = self.decl(v, ";")
            self.expect(";")
            return s + ";"
        if v == "if":
            self.next()
            cond = self.expr_until({"{"})
            s = f"if ({cond}) " + self.block(indent)
            while self.peek() == "else":
                self.next()
                if self.peek() == "if":
                    self.next()
                    cond = self.expr_until({"{"})
                    s += f" else if ({cond}) " + self.block(indent)
                else:
                    s += " else " + self.block(indent)
            return s
        if v == "for":
            self.next()
            self.expect("(")
            init = ""
            if self.peek() in ("var", "let"):
                kw = self.next()
                init = self.decl(kw, ";")
            elif self.peek() != ";":
                init = self.expr_until({";"})
            self.expect(";")
            cond = self.expr_until({";"})
            self.expect(";")
            step = self.expr_until({")"})
            self.expect(")")
            return f"for ({init}; {cond}; {step}) " + self.block(indent)
        if v == "while":
            self.next()
            cond = self.expr_until({"{"})
            return f"while ({cond}) " + self.block(indent)
        if v == "loop":
            self.next()
            return "for (;;) " + self.block(indent)
        if v == "{":
            return self.block(indent)
        if v in ("return", "break", "continue"):
            self.next()
            if v == "return" and self.peek() != ";":
                e = self.expr_until({";"})
                self.expect(";")
                return f"return {e};"
            self.expect(";")
            return v + ";"
        if v == ";":
            self.next()
            return ";"
        if v in UNSUPPORTED:
            raise WgslError(f"line {self.line()}: unsupported statement {v!r}")
        e = self.expr_until({";"})
        self.expect(";")
        return e + ";"

    # ---------------------------------------------------------------- module scope
    def run(self) -> str:
        while True:
            self.skip_nl()
            if self.i >= len(self.t):
                break
            attrs = self.skip_attributes()
            self.skip_nl()
            kw = self.next()
            if kw == "enable":
                self.expr_until({";"})
                self.expect(";")
            elif kw == "struct":
                self.struct()
            elif kw == "const":
                self.globals.append("static " + self.decl("const", ";") + ";")
                self.expect(";")
            elif kw == "override":
                name = self.ident(self.next())
                self.expect(":")
                ty = self.parse_type()
                init = "{}"
                if self.peek() == "=":
                    self.next()
                    init = "= " + self.expr_until({";"})
                self.expect(";")
                self.globals.append(f"{ty} {name} {init};  // pipeline-overridable: set by the harness")
            elif kw == "var":
                space = []
                if self.peek() == "<":
                    self.next()
                    while self.peek() != ">":
                        t = self.next()
                        if t != ",":
                            space.append(t)
                    self.next()
                name = self.ident(self.next())
                self.expect(":")
                ty = self.parse_type()
                if self.peek() == "=":
                    raise WgslError(f"line {self.line()}: initialised module-scope var")
                self.expect(";")
                prefix = "thread_local " if space[:1] == ["private"] else ""
                self.globals.append(f"{prefix}{ty} {name}{{}};  // {'<' + ', '.join(space) + '>' if space else ''}")
            elif kw == "fn":
                self.function(attrs)
            elif kw == ";":
                continue
            else:
                raise WgslError(f"line {self.line()}: unsupported module-scope item {kw!r}")
        out = [
            "// GENERATED by oracle/wgsl_translate.py from the reference's WGSL source.",
            "// Test infrastructure: never committed (oracle/_ref is git-ignored).",
            f"namespace {self.ns} {{",
            "using namespace wgsl_rt;",
            "",
        ]
        out += self.structs + [""] + self.globals + [""] + self.protos + [""] + self.bodies
        out.append(f"}}  // namespace {self.ns}")
        return "\n".join(out) + "\n"

    def struct(self):
        name = self.ident(self.next())
        self.expect("{")
        fields = []
        while True:
            self.skip_nl()
            if self.peek() == "}":
                self.next()
                break
            self.skip_attributes()
            f = self.ident(self.next())
            self.expect(":")
            ty = self.parse_type()
            fields.append(f"    {ty} {f}{{}};")
            if self.peek() == ",":
                self.next()
        if self.peek() == ";":
            self.next()
        self.structs.append(f"struct {name} {{\n" + "\n".join(fields) + "\n};")

    def function(self, attrs: list[str]):
        name = self.ident(self.next())
        self.expect("(")
        params = []
        while self.peek() != ")":
            self.skip_attributes()
            p = self.ident(self.next())
            self.expect(":")
            params.append(f"{self.parse_type()} {p}")
            if self.peek() == ",":
                self.next()
        self.expect(")")
        ret = "void"
        if self.peek() == "->":
            self.next()
            self.skip_attributes()
            ret = self.parse_type()
        sig = f"{ret} {name}({', '.join(params)})"
        self.protos.append(sig + ";")
        note = f"  // entry point ({', '.join(attrs)})" if attrs else ""
        self.bodies.append(sig + " " + self.block("") + note + "\n")


def main(argv):
    if len(argv) != 4:
        print(__doc__)
        return 2
    src = open(argv[1], encoding="utf-8").read()
    try:
        out = Translator(src, argv[3]).run()
    except WgslError as e:
        print(f"wgsl_translate: {argv[1]}: {e}", file=sys.stderr)
        return 1
    with open(argv[2], "w", encoding="utf-8") as f:
        f.write(out)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
