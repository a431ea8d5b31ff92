"""Source-to-source translator from the TypeScript subset of the reference's
host-side builders (src/lib/gpu/bvh.ts) to Python over oracle/js_rt.py.

TEST INFRASTRUCTURE ONLY: oracle/build_ref.py runs it on the reference
checkout at build time and writes the result under oracle/_ref/ (git-ignored),
so the reference's own builder can run here, where there is no JavaScript
runtime, and pin the restatement in oracle/bvh.py.

Supported: functions (typed parameters, return types), const / let / var
(several declarators, optional initialiser), interfaces and type aliases
(dropped), if / else, C-style for, for-of, while, return, break, continue,
the JavaScript operators with their precedence (bitwise ones through the
runtime's ToInt32 / ToUint32 helpers, `/` and `%` with IEEE results),
assignment operators, ++ / -- (as statements, in for updates, and post-
increments of a variable inside an expression), ?:, calls, member and index
access, `new`, array and object literals (with shorthand properties).
Module-level variables assigned inside functions become `global`s.  Block
scoping is not modelled: a name declared in an inner block shares the
function's Python scope, which is sound for code (like bvh.ts) that does not
read an outer binding after an inner one of the same name was declared.
"""
from __future__ import annotations

import keyword
import re

TS2PY_VERSION = "1"

_PUNCT = sorted("""
>>>= >>> === !== ... **= <<= >>= => <= >= == != && || ?? ?. ++ -- += -= *= /= %= |= &= ^= << >> **
{ } ( ) [ ] ; , < > + - * / % & | ^ ! ~ ? : = . @
""".split(), key=len, reverse=True)


class TsError(Exception):
    pass


class Tok:
    __slots__ = ("kind", "text", "line")

    def __init__(self, kind, text, line):
        self.kind, self.text, self.line = kind, text, line

    def __repr__(self):
        return f"{self.kind}:{self.text}@{self.line}"


def tokenize(src: str):
    out, i, line, n = [], 0, 1, len(src)
    while i < n:
        c = src[i]
        if c == "\n":
            line += 1
            i += 1
        elif c.isspace():
            i += 1
        elif src.startswith("//", i):
            while i < n and src[i] != "\n":
                i += 1
        elif src.startswith("/*", i):
            j = src.index("*/", i + 2)
            line += src.count("\n", i, j)
            i = j + 2
        elif c.isalpha() or c in "_$":
            j = i
            while j < n and (src[j].isalnum() or src[j] in "_$"):
                j += 1
            out.append(Tok("id", src[i:j], line))
            i = j
        elif c.isdigit() or (c == "." and i + 1 < n and src[i + 1].isdigit()):
            m = re.compile(r"0[xX][0-9a-fA-F_]+|(\d[\d_]*)?(\.\d[\d_]*)?([eE][+-]?\d+)?").match(src, i)
            out.append(Tok("num", m.group(0).replace("_", ""), line))
            i = m.end()
        elif c in "'\"`":
            j = i + 1
            while src[j] != c:
                j += 2 if src[j] == "\\" else 1
            out.append(Tok("str", src[i:j + 1], line))
            i = j + 1
        else:
            for p in _PUNCT:
                if src.startswith(p, i):
                    out.append(Tok("op", p, line))
                    i += len(p)
                    break
            else:
                raise TsError(f"line {line}: unexpected character {c!r}")
    out.append(Tok("eof", "", line))
    return out


# binary operators: precedence (higher binds tighter) and the Python form
_BIN = {
    "??": 3, "||": 3, "&&": 4, "|": 5, "^": 6, "&": 7,
    "==": 8, "!=": 8, "===": 8, "!==": 8,
    "<": 9, ">": 9, "<=": 9, ">=": 9,
    "<<": 10, ">>": 10, ">>>": 10,
    "+": 11, "-": 11, "*": 12, "/": 12, "%": 12,
}
_BIN_FN = {"|": "js_bor", "&": "js_band", "^": "js_bxor", "<<": "js_shl", ">>": "js_shr", ">>>": "js_ushr",
           "%": "js_mod", "/": "js_div"}
_BIN_PY = {"||": "or", "&&": "and", "==": "==", "!=": "!=", "===": "==", "!==": "!=",
           "<": "<", ">": ">", "<=": "<=", ">=": ">=", "+": "+", "-": "-", "*": "*"}
_ASSIGN = {"=", "+=", "-=", "*=", "/=", "%=", "|=", "&=", "^=", "<<=", ">>=", ">>>="}
_NAMES = {"Infinity": "Infinity", "NaN": "NaN", "undefined": "None", "null": "None", "true": "True",
          "false": "False"}


def _pyname(name: str) -> str:
    if name in _NAMES:
        return _NAMES[name]
    return name + "_" if keyword.iskeyword(name) or name in ("print", "len", "min", "max", "list") else name


class Translator:
    def __init__(self, src: str):
        self.t = tokenize(src)
        self.p = 0
        self.tmp = 0
        self.module_names: set = set()

    # -- token helpers
    def peek(self, k=0):
        return self.t[self.p + k]

    def next(self):
        tok = self.t[self.p]
        self.p += 1
        return tok

    def at(self, text, k=0):
        return self.t[self.p + k].text == text and self.t[self.p + k].kind in ("op", "id")

    def expect(self, text):
        tok = self.next()
        if tok.text != text:
            raise TsError(f"line {tok.line}: expected {text!r}, got {tok.text!r}")
        return tok

    def skip_type(self, stops):
        """Skips a type annotation up to one of `stops` at bracket depth 0."""
        depth = 0
        while True:
            tok = self.peek()
            if tok.kind == "eof":
                raise TsError("eof in type")
            if depth == 0 and tok.text in stops:
                return
            if tok.text in ("(", "[", "{", "<"):
                depth += 1
            elif tok.text in (")", "]", "}", ">"):
                depth -= 1
            self.next()

    def skip_balanced(self):
        """Skips `{ ... }`."""
        self.expect("{")
        depth = 1
        while depth:
            tok = self.next()
            if tok.text == "{":
                depth += 1
            elif tok.text == "}":
                depth -= 1

    # -- expressions: each returns the Python text; statements that must run first
    #    (hoisted post-increments) are appended to `pre`
    def expr(self, pre, min_prec=0):
        left = self.unary(pre)
        while True:
            tok = self.peek()
            if tok.kind != "op":
                return left
            op = tok.text
            if op == "?" and min_prec <= 2:
                self.next()
                a = self.expr(pre, 1)
                self.expect(":")
                b = self.expr(pre, 1)
                left = f"({a} if {left} else {b})"
                continue
            prec = _BIN.get(op)
            if prec is None or prec < min_prec or prec <= 2:
                return left
            self.next()
            right = self.expr(pre, prec + 1)
            if op in _BIN_FN:
                left = f"{_BIN_FN[op]}({left}, {right})"
            elif op == "??":
                left = f"({left} if {left} is not None else {right})"
            else:
                left = f"({left} {_BIN_PY[op]} {right})"

    def unary(self, pre):
        tok = self.peek()
        if tok.kind == "op" and tok.text in ("!", "-", "+", "~"):
            self.next()
            v = self.unary(pre)
            return {"!": f"(not {v})", "-": f"js_neg({v})", "+": f"(+{v})", "~": f"js_bnot({v})"}[tok.text]
        if tok.kind == "op" and tok.text in ("++", "--"):
            raise TsError(f"line {tok.line}: prefix {tok.text} inside an expression")
        if tok.kind == "id" and tok.text == "typeof":
            raise TsError(f"line {tok.line}: typeof")
        v = self.postfix(pre)
        if self.peek().kind == "op" and self.peek().text in ("++", "--"):
            op = self.next().text
            if not re.fullmatch(r"[A-Za-z_]\w*", v):
                raise TsError(f"line {tok.line}: {op} of a non-variable inside an expression")
            self.tmp += 1
            t = f"_pi{self.tmp}"
            pre.append(f"{t} = {v}")
            pre.append(f"{v} = {t} {'+' if op == '++' else '-'} 1")
            self.assigned.add(v)
            return t
        if self.peek().kind == "id" and self.peek().text == "as":
            self.next()
            self.skip_type((")", ",", ";", "]", "}"))
        return v

    def postfix(self, pre):
        v = self.primary(pre)
        while True:
            tok = self.peek()
            if tok.text == "." and tok.kind == "op":
                self.next()
                name = self.next().text
                v = f"{v}.{'from_' if name == 'from' else name}"
            elif tok.text == "[" and tok.kind == "op":
                self.next()
                i = self.expr(pre)
                self.expect("]")
                v = f"{v}[{i}]"
            elif tok.text == "(" and tok.kind == "op":
                self.next()
                v = f"{v}({', '.join(self.args(pre))})"
            elif tok.text == "!" and tok.kind == "op" and self.peek(1).text in (".", ")", ";", ",", "]", "["):
                self.next()  # non-null assertion
            else:
                return v

    def args(self, pre):
        out = []
        while not self.at(")"):
            out.append(self.expr(pre))
            if self.at(","):
                self.next()
        self.expect(")")
        return out

    def primary(self, pre):
        tok = self.next()
        if tok.kind == "num":
            s = tok.text
            if s.lower().startswith("0x"):
                return str(int(s, 16))
            return s if re.fullmatch(r"\d+", s) else repr(float(s))
        if tok.kind == "str":
            return repr(tok.text[1:-1])
        if tok.kind == "id":
            if tok.text == "new":
                ctor = self.next().text
                args = []
                if self.at("("):
                    self.next()
                    args = self.args(pre)
                return f"{_pyname(ctor)}({', '.join(args)})"
            if tok.text == "function":
                raise TsError(f"line {tok.line}: function expression")
            return _pyname(tok.text)
        if tok.text == "(":
            v = self.expr(pre)
            self.expect(")")
            return f"({v})"
        if tok.text == "[":
            items = []
            while not self.at("]"):
                items.append(self.expr(pre))
                if self.at(","):
                    self.next()
            self.expect("]")
            return f"JSArray([{', '.join(items)}])"
        if tok.text == "{":
            items = []
            while not self.at("}"):
                key = self.next().text
                if self.at(":"):
                    self.next()
                    items.append(f"{key}={self.expr(pre)}")
                else:
                    items.append(f"{key}={_pyname(key)}")
                if self.at(","):
                    self.next()
            self.expect("}")
            return f"JSObj({', '.join(items)})"
        raise TsError(f"line {tok.line}: unexpected {tok.text!r}")

    # -- statements: each returns a list of Python lines (unindented blocks nested by 4)
    def block_or_stmt(self):
        if self.at("{"):
            self.next()
            out = []
            while not self.at("}"):
                out += self.stmt()
            self.next()
            return out or ["pass"]
        return self.stmt() or ["pass"]

    def decl(self, top=False):
        self.next()  # const / let / var
        out = []
        while True:
            name = _pyname(self.next().text)
            if self.at(":"):
                self.next()
                self.skip_type(("=", ",", ";"))
            pre = []
            val = "None"
            if self.at("="):
                self.next()
                val = self.expr(pre)
            out += pre + [f"{name} = {val}"]
            if top:
                self.module_names.add(name)
            else:
                self.locals.add(name)
            if self.at(","):
                self.next()
                continue
            break
        if self.at(";"):
            self.next()
        return out

    def simple(self, pre, loop_update=False):
        """Assignment, ++/--, or a bare expression (no trailing `;`)."""
        start, tmp0 = self.p, self.tmp
        trial = []  # hoisted statements of the target, kept only if this is an assignment
        target = self.postfix(trial)
        tok = self.peek()
        if tok.kind == "op" and tok.text in ("++", "--"):
            self.next()
            self._note_assign(target)
            return pre + trial + [f"{target} {'+=' if tok.text == '++' else '-='} 1"]
        if tok.kind == "op" and tok.text in _ASSIGN:
            self.next()
            pre = pre + trial
            val = self.expr(pre)
            self._note_assign(target)
            op = tok.text
            if op == "=":
                return pre + [f"{target} = {val}"]
            base = op[:-1]
            if base in _BIN_FN:
                return pre + [f"{target} = {_BIN_FN[base]}({target}, {val})"]
            return pre + [f"{target} {op} {val}"]
        self.p, self.tmp = start, tmp0
        v = self.expr(pre)
        return pre + [v]

    def _note_assign(self, target):
        if re.fullmatch(r"[A-Za-z_]\w*", target):
            self.assigned.add(target)

    def stmt(self):
        tok = self.peek()
        if tok.text == ";":
            self.next()
            return []
        if tok.kind == "id" and tok.text in ("const", "let", "var"):
            return self.decl()
        if tok.kind == "id" and tok.text == "return":
            self.next()
            if self.at(";") or self.at("}"):
                if self.at(";"):
                    self.next()
                return ["return None"]
            pre = []
            v = self.expr(pre)
            if self.at(";"):
                self.next()
            return pre + [f"return {v}"]
        if tok.kind == "id" and tok.text in ("break", "continue"):
            self.next()
            if self.at(";"):
                self.next()
            if tok.text == "continue" and self.loop_updates and self.loop_updates[-1]:
                return list(self.loop_updates[-1]) + ["continue"]
            return [tok.text]
        if tok.kind == "id" and tok.text == "if":
            self.next()
            self.expect("(")
            pre = []
            cond = self.expr(pre)
            self.expect(")")
            body = self.block_or_stmt()
            out = pre + [f"if {cond}:"] + ["    " + x for x in body]
            if self.at("else"):
                self.next()
                eb = self.block_or_stmt()
                out += ["else:"] + ["    " + x for x in eb]
            return out
        if tok.kind == "id" and tok.text == "while":
            self.next()
            self.expect("(")
            pre = []
            cond = self.expr(pre)
            if pre:
                raise TsError(f"line {tok.line}: side effects in a loop condition")
            self.expect(")")
            self.loop_updates.append(None)
            body = self.block_or_stmt()
            self.loop_updates.pop()
            return [f"while {cond}:"] + ["    " + x for x in body]
        if tok.kind == "id" and tok.text == "for":
            return self.for_stmt()
        if tok.kind == "id" and tok.text in ("interface", "type"):
            self.next()
            self.next()
            if tok.text == "type":
                self.skip_type((";",))
                self.next()
            else:
                self.skip_balanced()
            return []
        pre = []
        out = self.simple(pre)
        if self.at(";"):
            self.next()
        return out

    def for_stmt(self):
        line = self.next().line
        self.expect("(")
        if self.at("const") or self.at("let") or self.at("var"):
            if self.peek(2).text == "of":
                self.next()
                name = _pyname(self.next().text)
                self.locals.add(name)
                self.next()  # of
                pre = []
                it = self.expr(pre)
                self.expect(")")
                self.loop_updates.append(None)
                body = self.block_or_stmt()
                self.loop_updates.pop()
                return pre + [f"for {name} in {it}:"] + ["    " + x for x in body]
            init = self.decl()
        elif self.at(";"):
            self.next()
            init = []
        else:
            init = self.simple([])
            self.expect(";")
        pre = []
        cond = "True" if self.at(";") else self.expr(pre)
        if pre:
            raise TsError(f"line {line}: side effects in a loop condition")
        self.expect(";")
        update = [] if self.at(")") else self.simple([])
        self.expect(")")
        self.loop_updates.append(update)
        body = self.block_or_stmt()
        self.loop_updates.pop()
        return init + [f"while {cond}:"] + ["    " + x for x in body + update]

    def function(self):
        self.expect("function")
        name = _pyname(self.next().text)
        self.expect("(")
        params = []
        while not self.at(")"):
            pname = _pyname(self.next().text)
            if self.at("?"):
                self.next()
            default = None
            if self.at(":"):
                self.next()
                self.skip_type((",", ")", "="))
            if self.at("="):
                self.next()
                default = self.expr([])
            params.append(f"{pname}={default}" if default is not None else f"{pname}=None")
            if self.at(","):
                self.next()
        self.expect(")")
        if self.at(":"):
            self.next()
            self.skip_type(("{",))
        self.locals = {p.split("=")[0] for p in params}
        self.assigned = set()
        self.loop_updates = []
        self.expect("{")
        body = []
        while not self.at("}"):
            body += self.stmt()
        self.next()
        globs = sorted((self.assigned & self.module_names) - self.locals)
        head = [f"def {name}({', '.join(params + ['*_extra'])}):"]  # JS ignores surplus arguments
        if globs:
            head.append(f"    global {', '.join(globs)}")
        self.module_names.add(name)
        return head + ["    " + x for x in (body or ["pass"])] + [""]

    def module(self, origin: str) -> str:
        out = [f"# Translated by oracle/ts2py.py (version {TS2PY_VERSION}) from {origin}; do not edit.",
               "from js_rt import *  # noqa: F401,F403", ""]
        self.locals, self.assigned, self.loop_updates = set(), set(), []
        while self.peek().kind != "eof":
            tok = self.peek()
            if tok.kind == "id" and tok.text == "export":
                self.next()
                continue
            if tok.kind == "id" and tok.text == "import":
                while not self.at(";"):
                    self.next()
                self.next()
                continue
            if tok.kind == "id" and tok.text == "function":
                out += self.function()
                continue
            if tok.kind == "id" and tok.text in ("const", "let", "var"):
                out += self.decl(top=True)
                continue
            out += self.stmt()
        return "\n".join(out) + "\n"


def translate(src: str, origin: str) -> str:
    return Translator(src).module(origin)
