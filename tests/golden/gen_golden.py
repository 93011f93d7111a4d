#!/usr/bin/env python3
"""Extract the reference's own known-answer test vectors into JSON fixtures.

Run once in a container that has the reference source tree; the fixtures it
writes next to this script are committed, and nothing at test time reads the
reference.  Usage:  python tests/golden/gen_golden.py REFERENCE_ROOT

The reference keeps its test vectors as Rust literals inside `#[cfg(test)]`
modules.  This script tokenises those literal arrays with a small expression
evaluator (integers with suffixes, `+ - * << >> & |`, tuples, `vec![..]`,
`vec![x; n]`, ranges with `.map/.chain/.collect`, `Some/None`, struct
literals and the test helpers `str_to_quants`/`str_to_bools`) and writes:

  quant_reducer.json        qsat.rs:2036-2466  test_quant_reducer
  aggr_tree_cpu.json        qsat.rs:2629-2835  test_aggr_output_cpu_code
  aggr_tree_opencl.json     qsat.rs:3434-3520  test_aggr_output_opencl_code
  aggr_tree_cpu_words.json  qsat.rs:2837-3292  test_aggr_output_cpu_code_2
  aggr_tree_opencl_groups.json qsat.rs:3522-3857 test_aggr_output_opencl_code_2
  final_result_circuit.json qsat.rs:6033-6267  final_result_with_circuit
  opencl_quant_reducer.json qsat.rs:4038-6008  test_opencl_quant_reducer
  cpu_outputs_final_result.json qsat.rs:3859-4036
                            test_get_final_results_from_cpu_outputs
  greedy_find_solution.json greedysatostop.rs:1204-1268
  greedy_mem_image.json     greedysatostop.rs:1145-1201
  greedy_file_image.json    greedysatostop.rs:1271-1354
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


# --------------------------------------------------------------------------
# tokenizer / evaluator for the Rust literal subset used by the tests

TOKEN_RE = re.compile(
    r"""\s*(?:
        (?P<str>"(?:[^"\\]|\\.)*")
      | (?P<num>0x[0-9a-fA-F_]+|0b[01_]+|[0-9][0-9_]*)(?P<suf>u8|u16|u32|u64|u128|usize|i32|i64)?
      | (?P<id>[A-Za-z_][A-Za-z0-9_]*)
      | (?P<op>::|\.\.|<<|>>|=>|==|!=|[()\[\]{},;:&|+\-*.!<>_?=])
    )""",
    re.VERBOSE,
)


def tokenize(src):
    toks = []
    pos = 0
    while True:
        # skip comments
        while True:
            m = re.match(r"\s*//[^\n]*", src[pos:])
            if m and m.group(0).strip():
                pos += m.end()
                continue
            break
        if pos >= len(src) or not src[pos:].strip():
            break
        m = TOKEN_RE.match(src, pos)
        if not m:
            raise ValueError("cannot tokenize at: %r" % src[pos:pos + 40])
        pos = m.end()
        if m.group("str") is not None:
            toks.append(("str", bytes(m.group("str")[1:-1], "utf-8").decode("unicode_escape")))
        elif m.group("num") is not None:
            t = m.group("num").replace("_", "")
            v = int(t, 16) if t.startswith("0x") else int(t, 2) if t.startswith("0b") else int(t)
            toks.append(("num", v))
        elif m.group("id") is not None:
            toks.append(("id", m.group("id")))
        else:
            toks.append(("op", m.group("op")))
    toks.append(("eof", None))
    return toks


class Repeat:
    def __init__(self, value):
        self.value = value


class Closure:
    def __init__(self, param, body, parser, env=None):
        self.param, self.body, self.parser, self.env = param, body, parser, dict(env or {})

    def __call__(self, x):
        return self.parser.eval_ast(self.body, dict(self.env, **{self.param: x}))


def str_to_quants(s):
    return "".join(c.upper() for c in s if c.lower() in "ae")


def str_to_bools(s):
    return [1 if c == "1" else 0 for c in s if c in "01"]


class Parser:
    """Builds a tiny AST and evaluates it; binary precedence follows Rust."""

    PREC = [("==", "!="), ("|",), ("^",), ("&",), ("<<", ">>"), ("+", "-"), ("*",)]

    def __init__(self, src):
        self.t = tokenize(src)
        self.i = 0

    def peek(self, k=0):
        return self.t[self.i + k]

    def take(self, kind=None, val=None):
        tok = self.t[self.i]
        if kind and tok[0] != kind or val is not None and tok[1] != val:
            raise ValueError("expected %s %s got %s near %s" % (kind, val, tok, self.t[self.i:self.i + 6]))
        self.i += 1
        return tok

    def is_op(self, v, k=0):
        tok = self.peek(k)
        return tok[0] == "op" and tok[1] == v

    # expressions -> AST tuples
    def expr(self, level=0):
        if level == len(self.PREC):
            return self.unary()
        lhs = self.expr(level + 1)
        while self.peek()[0] == "op" and self.peek()[1] in self.PREC[level]:
            # `|` directly followed by an identifier and `|` is a closure, not here
            op = self.take()[1]
            rhs = self.expr(level + 1)
            lhs = ("bin", op, lhs, rhs)
        if level == 0 and self.is_op(".."):
            self.take()
            rhs = self.expr(0)
            lhs = ("range", lhs, rhs)
        return lhs

    def unary(self):
        if self.is_op("&"):
            self.take()
            return self.unary()
        if self.is_op("-"):
            self.take()
            return ("neg", self.unary())
        node = self.postfix(self.primary())
        while self.peek() == ("id", "as"):       # `as u16`: truncation to the type
            self.take()
            node = ("cast", self.take("id")[1], node)
        return node

    def postfix(self, node):
        while self.is_op("."):
            self.take()
            name = self.take("id")[1]
            if self.is_op("::"):  # turbofish ::<Vec<_>>
                self.take()
                depth = 0
                while True:
                    tok = self.take()
                    if tok == ("op", "<"):
                        depth += 1
                    elif tok == ("op", ">"):
                        depth -= 1
                        if depth == 0:
                            break
                    elif tok == ("op", ">>"):
                        depth -= 2
                        if depth <= 0:
                            break
            self.take("op", "(")
            args = []
            while not self.is_op(")"):
                args.append(self.closure_or_expr())
                if self.is_op(","):
                    self.take()
            self.take("op", ")")
            node = ("method", name, node, args)
        return node

    def closure_or_expr(self):
        if self.is_op("|"):
            self.take()
            param = self.take("id")[1]
            self.take("op", "|")
            return ("closure", param, self.expr())
        return self.expr()

    def block(self):
        """`{ expr }`: a block whose value is its one expression."""
        self.take("op", "{")
        e = self.expr()
        self.take("op", "}")
        return e

    def seq(self, close):
        items = []
        while not self.is_op(close):
            items.append(self.expr())
            if self.is_op(","):
                self.take()
            elif self.is_op(";"):
                self.take()
                count = self.expr()
                self.take("op", close)
                return ("repeat", items[0], count)
        self.take("op", close)
        return ("list", items)

    def primary(self):
        tok = self.peek()
        if tok[0] == "num":
            self.take()
            return ("lit", tok[1])
        if tok[0] == "str":
            self.take()
            return ("lit", tok[1])
        if self.is_op("("):
            self.take()
            if self.is_op(")"):
                self.take()
                return ("tuple", [])
            first = self.expr()
            if self.is_op(")"):
                self.take()
                return first
            items = [first]
            while self.is_op(","):
                self.take()
                if self.is_op(")"):
                    break
                items.append(self.expr())
            self.take("op", ")")
            return ("tuple", items)
        if self.is_op("["):
            self.take()
            return self.seq("]")
        if self.is_op("{"):
            return self.block()
        if tok == ("id", "if"):
            self.take()
            cond = self.expr()
            then = self.block()
            self.take("id", "else")
            other = self.block() if self.is_op("{") else self.primary()
            return ("if", cond, then, other)
        if tok[0] == "id":
            name = self.take()[1]
            # path segments: Option::<FinalResult>::None, std::iter::...
            while self.is_op("::"):
                self.take()
                if self.is_op("<"):
                    depth = 0
                    while True:
                        t2 = self.take()
                        if t2 == ("op", "<"):
                            depth += 1
                        elif t2 == ("op", ">"):
                            depth -= 1
                            if depth == 0:
                                break
                    self.take("op", "::")
                name = self.take("id")[1]
            if name in ("true", "false"):
                return ("lit", name == "true")
            if name == "None":
                return ("lit", None)
            if self.is_op("!"):  # macro
                self.take()
                if self.is_op("["):
                    self.take()
                    return self.seq("]")
                self.take("op", "(")
                args = []
                while not self.is_op(")"):
                    args.append(self.expr())
                    if self.is_op(","):
                        self.take()
                self.take("op", ")")
                return ("call", name + "!", args)
            if self.is_op("{"):  # struct literal
                self.take()
                fields = {}
                while not self.is_op("}"):
                    key = self.take("id")[1]
                    self.take("op", ":")
                    fields[key] = self.expr()
                    if self.is_op(","):
                        self.take()
                self.take("op", "}")
                return ("struct", name, fields)
            if self.is_op("("):
                self.take()
                args = []
                while not self.is_op(")"):
                    args.append(self.expr())
                    if self.is_op(","):
                        self.take()
                self.take("op", ")")
                return ("call", name, args)
            return ("var", name)
        raise ValueError("unexpected token %s near %s" % (tok, self.t[self.i:self.i + 8]))

    def eval_ast(self, n, env=None):
        env = env or {}
        k = n[0]
        if k == "lit":
            return n[1]
        if k == "var":
            # enum variants and statics (CPUExtension::NoExtension, CLANG_WRITER_U64)
            # evaluate to their own name
            return env.get(n[1], n[1])
        if k == "neg":
            return -self.eval_ast(n[1], env)
        if k == "if":
            return self.eval_ast(n[2] if self.eval_ast(n[1], env) else n[3], env)
        if k == "cast":
            bits = {"u8": 8, "u16": 16, "u32": 32, "u64": 64, "u128": 128, "usize": 64}[n[1]]
            return self.eval_ast(n[2], env) & ((1 << bits) - 1)
        if k == "bin":
            a, b = self.eval_ast(n[2], env), self.eval_ast(n[3], env)
            return {"==": lambda: a == b, "!=": lambda: a != b,
                    "|": lambda: a | b, "^": lambda: a ^ b, "&": lambda: a & b,
                    "<<": lambda: a << b, ">>": lambda: a >> b, "+": lambda: a + b,
                    "-": lambda: a - b, "*": lambda: a * b}[n[1]]()
        if k == "range":
            return list(range(self.eval_ast(n[1], env), self.eval_ast(n[2], env)))
        if k == "tuple":
            return tuple(self.eval_ast(x, env) for x in n[1])
        if k == "list":
            return [self.eval_ast(x, env) for x in n[1]]
        if k == "repeat":
            return [self.eval_ast(n[1], env)] * self.eval_ast(n[2], env)
        if k == "closure":
            return Closure(n[1], n[2], self, env)
        if k == "struct":
            return dict(_type=n[1], **{f: self.eval_ast(v, env) for f, v in n[2].items()})
        if k == "call":
            args = [self.eval_ast(a, env) for a in n[2]]
            name = n[1]
            if name == "str_to_quants":
                return str_to_quants(args[0])
            if name == "str_to_bools":
                return str_to_bools(args[0])
            if name == "concat!":
                return "".join(args)
            if name == "Some":
                return args[0]
            if name == "repeat":          # iter::repeat(x): unbounded until .take(n)
                return Repeat(args[0])
            if name == "once":            # iter::once(x)
                return [args[0]]
            raise ValueError("unknown call " + name)
        if k == "method":
            name, base = n[1], self.eval_ast(n[2], env)
            args = [self.eval_ast(a, env) for a in n[3]]
            if name in ("collect", "into_iter", "iter", "to_vec"):
                return list(base)
            if name == "chain":
                return list(base) + list(args[0])
            if name == "map":
                return [args[0](x) for x in base]
            if name == "flatten":
                return [x for part in base for x in part]
            if name == "rotate_left":         # the tests rotate u64 literals
                r = args[0] % 64
                return ((base << r) | (base >> (64 - r))) & ((1 << 64) - 1)
            if name == "take":
                return [base.value] * args[0] if isinstance(base, Repeat) else list(base)[:args[0]]
            raise ValueError("unknown method " + name)
        raise ValueError("bad node %r" % (k,))


def rle(values):
    out = []
    for v in values:
        if out and out[-1][0] == v:
            out[-1][1] += 1
        else:
            out.append([v, 1])
    return out


def fn_body(src, name):
    start = src.index("fn %s(" % name)
    i = src.index("{", start)
    depth = 0
    for j in range(i, len(src)):
        if src[j] == "{":
            depth += 1
        elif src[j] == "}":
            depth -= 1
            if depth == 0:
                return src[i:j + 1], src[:start].count("\n") + 1
    raise ValueError(name)


def case_array(body, anchor="in ["):
    """The literal array that follows the first `in [` of the test body."""
    m = re.search(r"\bin\s*\[", body)
    if not m:
        raise ValueError("no case array")
    start = m.end() - 1
    depth = 0
    for j in range(start, len(body)):
        c = body[j]
        if c == "[":
            depth += 1
        elif c == "]":
            depth -= 1
            if depth == 0:
                return body[start:j + 1]
    raise ValueError("no array")


def parse_cases(body, anchor="in ["):
    p = Parser(case_array(body, anchor))
    return p.eval_ast(p.primary())


def final_result(d):
    return {"reversed": bool(d["reversed"]), "solution_bits": d["solution_bits"],
            "solution": d["solution"]}


def main():
    if len(sys.argv) < 2:
        raise SystemExit("usage: gen_golden.py <root of the reference's source tree>")
    ref = sys.argv[1]
    qsat = open(os.path.join(ref, "src/qsat.rs")).read()
    greedy = open(os.path.join(ref, "src/greedysatostop.rs")).read()
    out = {}

    body, line = fn_body(qsat, "test_quant_reducer")
    cases = []
    for (quants, items, ordering, push_index, result) in parse_cases(body):
        cases.append({"quants": quants, "items": items, "ordering": ordering,
                      "push_index": push_index, "result": final_result(result)})
    out["quant_reducer.json"] = {"source": "src/qsat.rs:%d test_quant_reducer" % line, "cases": cases}

    body, line = fn_body(qsat, "test_aggr_output_cpu_code")
    cases = []
    for (exts, writer, quants, tests) in parse_cases(body):
        for (words, result) in tests:
            cases.append({"quants": quants, "words": words, "result": bool(result),
                          "cpu_type": "x".join(str(e) for e in [len(words) * 32])})
    out["aggr_tree_cpu.json"] = {"source": "src/qsat.rs:%d test_aggr_output_cpu_code" % line,
                                 "note": "item i = bit (i % 32) of word i // 32; result = full "
                                         "quantifier tree over all items",
                                 "cases": cases}

    body, line = fn_body(qsat, "test_aggr_output_cpu_code_2")
    cases = []
    for (elem_bits, quants, tests) in parse_cases(body):
        for (data, mword, found, result) in tests:
            cases.append({"elem_bits": elem_bits, "quants": quants, "data": data, "mword": mword,
                          "found": found, "result": bool(result)})
    out["aggr_tree_cpu_words.json"] = {
        "source": "src/qsat.rs:%d test_aggr_output_cpu_code_2" % line,
        "note": "identity circuit over data: item k = bit k%32 of data[k/32], 2^elem_bits items, 64-bit "
                "machine words (TYPE_LEN 64); result = the call's value over the last elem_bits quantifiers; "
                "found = index of the first deciding machine word (not bit-reversed), mword its value",
        "cases": cases}

    body, line = fn_body(qsat, "test_aggr_output_opencl_code_2")
    cases = []
    for (quants, group_len, reduce_len, tests) in parse_cases(body):
        for (data, results) in tests:
            cases.append({"quants": quants, "group_len": group_len, "reduce_len": reduce_len, "data": data,
                          "results": [[bool(r), l] for (r, l) in results]})
    out["aggr_tree_opencl_groups.json"] = {
        "source": "src/qsat.rs:%d test_aggr_output_opencl_code_2" % line,
        "note": "identity circuit over data: each of reduce_len groups is group_len 32-lane words (item k of a "
                "group = bit k%32 of its word k/32) under the last log2(group_len)+5 quantifiers; results: per "
                "group the value and the local index of the first decisive unit's word (0x7fff none, null "
                "unchecked)",
        "cases": cases}

    body, line = fn_body(qsat, "test_aggr_output_opencl_code")
    cases = []
    for (quants, tests) in parse_cases(body):
        for (words, result, lidx) in tests:
            cases.append({"quants": quants, "words": words, "result": bool(result)})
    out["aggr_tree_opencl.json"] = {"source": "src/qsat.rs:%d test_aggr_output_opencl_code" % line,
                                    "note": "one 32-lane word; result = tree over the last 5 "
                                            "quantifiers (TYPE_QUANT_REDUCE_OP_0..4)",
                                    "cases": cases}

    body, line = fn_body(qsat, "test_opencl_quant_reducer_final_result_with_circuit")
    cases = []
    for (rsb, reb, iglb, quants, group_len, tests) in parse_cases(body):
        fq = quants[0]
        fqb = len(quants) - len(quants.lstrip(fq)) - rsb
        solution_bits = min(reb + iglb, rsb + fqb)
        for (solution, values, exp) in tests:
            cases.append({"quants": quants, "circuit_solution_bits": solution_bits,
                          "solution": solution, "values": values, "expected": final_result(exp)})
    out["final_result_circuit.json"] = {
        "source": "src/qsat.rs:%d test_opencl_quant_reducer_final_result_with_circuit" % line,
        "note": "circuit = booltable(inputs[sb..sb+5], values) AND inputs[0..sb]==solution "
                "(gen_circuit, qsat.rs:6010-6030); the expected value completes the first-"
                "quantifier bits below sb from the circuit with inputs[0..sb] fixed",
        "cases": cases}

    body, line = fn_body(qsat, "test_opencl_quant_reducer")
    cases = []
    for k, (rsb, reb, iglb, quants, group_len, tests) in enumerate(parse_cases(body)):
        for (inputs, (exp, value)) in tests:
            cases.append({"case": k, "reduce_start_bit": rsb, "reduce_end_bit": reb, "init_group_len_bits": iglb,
                          "quants": quants, "group_len": group_len, "inputs_rle": rle(inputs),
                          "expected": None if exp is None else final_result(exp), "value": bool(value)})
    out["opencl_quant_reducer.json"] = {
        "source": "src/qsat.rs:%d test_opencl_quant_reducer" % line,
        "note": "inputs: one u16 per group of the bits reduce_end_bit..reduce_end_bit+init_group_len_bits "
                "(bit 15 the group's value, bits 0..14 the group-local index of the first decisive unit, "
                "0x7fff none), groups in index order over bits reduce_start_bit..reduce_end_bit, stored as "
                "[value, run length] pairs; expected: "
                "the reducer's FinalResult (None when it has none) and the formula's value",
        "cases": cases}

    body, line = fn_body(qsat, "test_get_final_results_from_cpu_outputs")
    cases = []
    for m in re.finditer(r"assert_eq!\(", body):
        i, depth = m.end() - 1, 0
        for j in range(i, len(body)):
            depth += {"(": 1, ")": -1}.get(body[j], 0)
            if depth == 0:
                break
        call = body[i + 1:j]
        k = call.index("get_final_results_from_cpu_outputs(")
        exp, value = Parser(call[:k].rstrip().rstrip(",")).eval_ast(Parser(call[:k].rstrip().rstrip(",")).primary())
        args = call[k + len("get_final_results_from_cpu_outputs("):]
        type_len, elem_bits = (int(x) for x in re.findall(r"\d+", args)[:2])
        quants = str_to_quants(re.search(r'str_to_quants\("([^"]*)"\)', args).group(1))
        arr = args[args.index("&[") + 1:args.rindex("[..]")]
        p2 = Parser(arr)
        outputs = p2.eval_ast(p2.primary())
        cases.append({"type_len": type_len, "elem_bits": elem_bits, "quants": quants, "outputs": outputs,
                      "expected": None if exp is None else final_result(exp), "value": bool(value)})
    out["cpu_outputs_final_result.json"] = {
        "source": "src/qsat.rs:%d test_get_final_results_from_cpu_outputs" % line,
        "note": "outputs: words 0..type_len/32 the lane values of the deciding word, then the call's value, "
                "a solution flag and the deciding word's index (low, high) within the call; expected: the "
                "FinalResult of the call's part of the formula (None when it has none) and the call's value",
        "cases": cases}

    body, line = fn_body(greedy, "test_mem_image_find_solution")
    cases = []
    for (state_len, start, ln, unknowns, pos_sol, nxt, exp) in parse_cases(body):
        cases.append({"state_len": state_len, "start": start, "len": ln, "unknowns": unknowns,
                      "pos_sol": pos_sol, "next": nxt,
                      "expected": None if exp is None else {"start": exp["start"], "end": exp["end"]}})
    out["greedy_find_solution.json"] = {"source": "src/greedysatostop.rs:%d" % line, "cases": cases}

    body, line = fn_body(greedy, "test_mem_image")
    cases = [{"state_len": a, "mult": b, "add": c, "len": d} for (a, b, c, d) in parse_cases(body)]
    out["greedy_mem_image.json"] = {
        "source": "src/greedysatostop.rs:%d" % line,
        "note": "entry i = (i * mult + add) mod 2^64 masked to state_len+1 bits; bit b of entry i "
                "lives at bit (i*(state_len+1)+b) of the u64 word array",
        "cases": cases}

    body, line = fn_body(greedy, "test_file_image")
    cases = [{"state_len": a, "mult": b, "add": c, "partitions": d, "changer": e}
             for (a, b, c, d, e) in parse_cases(body)]
    out["greedy_file_image.json"] = {"source": "src/greedysatostop.rs:%d" % line, "cases": cases}

    for name, obj in out.items():
        with open(os.path.join(HERE, name), "w") as f:
            json.dump(obj, f, indent=1)
            f.write("\n")
        print(name, len(obj["cases"]), "cases")


if __name__ == "__main__":
    main()
