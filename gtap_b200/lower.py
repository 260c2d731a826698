"""Source-to-source lowering of `#pragma gtap` programs to the task ABI.

The reference's compiler front end (clang-gtap) is not part of its checkout,
so programs written with the pragmas of examples/README.md:70-79 cannot be
built from it.  This module lowers the same pragmas, for a restricted subset
of C++, into the switch state machines the task ABI expects
(include/gtap_thread.cuh, include/gtap_block.cuh), which nvcc then compiles:

    python -m gtap_b200.lower prog.cu -o prog_lowered.cu [--mode thread|block]

Pragmas
  #pragma gtap function               before a `__device__ T name(params) {...}`
  #pragma gtap task [queue(expr)]     before `name(args);` or `lhs = name(args);`
  #pragma gtap taskwait [queue(expr)] waits for the children spawned since the last one
  #pragma gtap entry                  in a __global__ kernel, before `[lhs =] name(args);`

Lowering (the contract of the reference's task ABI):
  * each task function becomes `void name__gtap_task(void*, int, TaskContext*)`
    with a frame struct `__gtap_frame_name` holding its parameters, the
    locals declared at the top level of its body, the return value
    (`__ret`) and one child id per spawn site whose result is used;
  * the body is split at its taskwaits into the cases of a switch on
    __gtap_get_task_state; a taskwait becomes __gtap_set_state_for_join
    (thread mode) or __gtap_set_state_for_join_block (block mode) and returns
    when children are outstanding;
  * a spawn becomes __gtap_spawn_task with the arguments written into the
    child's frame; a child whose result is assigned is retained, and its
    result is read from its frame, and its id released, right after the
    taskwait that joins it;
  * `return e;` stores e in the frame and calls __gtap_finish_task;
  * an entry pushes the root as task 0 (through a small entry task when its
    result is assigned) and runs __gtap_execute_task_loop_device.

Restrictions (reported as LoweringError with the line):
  * taskwaits at the top level of a task function's body (not inside if/for);
  * locals that live across a taskwait declared at the top level of the body,
    with builtin arithmetic or pointer types, no arrays, no shadowing;
  * a spawn whose result is assigned is not inside a loop, and a taskwait
    follows it;
  * task functions are only called through `#pragma gtap task` / `entry`.
"""
import argparse
import re
import sys

class LoweringError(Exception):
    pass


# ---------------------------------------------------------------------------
# lexical helpers (strings, characters and comments are skipped)
# ---------------------------------------------------------------------------
def _skip_literal(src, i):
    """Index after the string/char literal or comment starting at i, or i."""
    c = src[i]
    if src.startswith("//", i):
        j = src.find("\n", i)
        return len(src) if j < 0 else j
    if src.startswith("/*", i):
        j = src.find("*/", i + 2)
        return len(src) if j < 0 else j + 2
    if c in "\"'":
        j = i + 1
        while j < len(src) and src[j] != c:
            j += 2 if src[j] == "\\" else 1
        return j + 1
    return i


def match_close(src, i, open_ch="{", close_ch="}"):
    """Index of the bracket closing the one at src[i]."""
    depth = 0
    j = i
    while j < len(src):
        k = _skip_literal(src, j)
        if k != j:
            j = k
            continue
        if src[j] == open_ch:
            depth += 1
        elif src[j] == close_ch:
            depth -= 1
            if depth == 0:
                return j
        j += 1
    raise LoweringError("unbalanced '%s' at line %d" % (open_ch, line_of(src, i)))


def line_of(src, i):
    return src.count("\n", 0, i) + 1


def split_top(s, sep=","):
    """Split at top-level separators (outside (), [], {})."""
    out, depth, cur, j = [], 0, [], 0
    while j < len(s):
        k = _skip_literal(s, j)
        if k != j:
            cur.append(s[j:k])
            j = k
            continue
        c = s[j]
        if c in "([{":
            depth += 1
        elif c in ")]}":
            depth -= 1
        if c == sep and depth == 0:
            out.append("".join(cur))
            cur = []
        else:
            cur.append(c)
        j += 1
    if "".join(cur).strip():
        out.append("".join(cur))
    return [x.strip() for x in out]


def statement_end(src, i):
    """Index of the ';' ending the statement starting at i (outside brackets)."""
    depth = 0
    j = i
    while j < len(src):
        k = _skip_literal(src, j)
        if k != j:
            j = k
            continue
        c = src[j]
        if c in "([{":
            depth += 1
        elif c in ")]}":
            depth -= 1
        elif c == ";" and depth == 0:
            return j
        j += 1
    raise LoweringError("statement at line %d has no ';'" % line_of(src, i))


def replace_identifiers(text, names, prefix="__f->"):
    """prefix every identifier in `names` that is not a member (after . or ->)."""
    out, j = [], 0
    ident = re.compile(r"[A-Za-z_]\w*")
    while j < len(text):
        k = _skip_literal(text, j)
        if k != j:
            out.append(text[j:k])
            j = k
            continue
        m = ident.match(text, j)
        if m:
            w = m.group(0)
            before = "".join(out).rstrip()
            if w in names and not before.endswith(".") and not before.endswith("->"):
                out.append(prefix + w)
            else:
                out.append(w)
            j = m.end()
            continue
        out.append(text[j])
        j += 1
    return "".join(out)


PRAGMA = re.compile(r"^[ \t]*#[ \t]*pragma[ \t]+gtap[ \t]+(\w+)(.*)$", re.M)
PRAGMA_AT = re.compile(r"#[ \t]*pragma[ \t]+gtap[ \t]+(\w+)(.*)$", re.M)   # at a known '#' 


def parse_queue(rest, line):
    rest = rest.strip()
    if not rest:
        return None
    m = re.match(r"queue\s*\((.*)\)\s*$", rest)
    if not m:
        raise LoweringError("line %d: unknown pragma clause '%s'" % (line, rest))
    return m.group(1).strip()


# ---------------------------------------------------------------------------
# task functions
# ---------------------------------------------------------------------------
class Param:
    def __init__(self, ctype, name):
        self.ctype, self.name = ctype, name


def parse_params(text, line):
    params = []
    for p in split_top(text):
        if not p or p == "void":
            continue
        m = re.match(r"^(.*?)([A-Za-z_]\w*)\s*$", p, re.S)
        if not m or "[" in p:
            raise LoweringError("line %d: unsupported parameter '%s'" % (line, p))
        params.append(Param(" ".join(m.group(1).split()), m.group(2)))
    return params


class TaskFunction:
    def __init__(self, name, ret, params, body, start, end, line):
        self.name, self.ret, self.params, self.body = name, ret, params, body
        self.start, self.end, self.line = start, end, line
        self.locals = []        # [Param]
        self.child_slots = []   # names of child-id fields

    @property
    def frame(self):
        return "__gtap_frame_" + self.name

    @property
    def task(self):
        return self.name + "__gtap_task"


FUNC_SIG = re.compile(r"\s*((?:(?:__device__|__forceinline__|__noinline__|static|inline)\s+)*)"
                      r"([A-Za-z_][\w\s\*:<>,]*?)\s*\b([A-Za-z_]\w*)\s*\(")


def find_functions(src):
    funcs = []
    for m in PRAGMA.finditer(src):
        if m.group(1) != "function":
            continue
        s = m.end()
        sig = FUNC_SIG.match(src, s)
        if not sig:
            raise LoweringError("line %d: '#pragma gtap function' is not followed by a function" % line_of(src, s))
        if "__device__" not in sig.group(1):
            raise LoweringError("line %d: a task function must be __device__" % line_of(src, s))
        po = sig.end() - 1
        pc = match_close(src, po, "(", ")")
        bo = src.index("{", pc)
        if src[pc + 1:bo].strip():
            raise LoweringError("line %d: unexpected text before the function body" % line_of(src, pc))
        bc = match_close(src, bo)
        funcs.append(TaskFunction(sig.group(3), " ".join(sig.group(2).split()),
                                  parse_params(src[po + 1:pc], line_of(src, po)), src[bo + 1:bc],
                                  m.start(), bc + 1, line_of(src, m.start())))
    return funcs


def top_level_statements(body):
    """(start, end) of each statement or pragma line at brace depth 0."""
    out, j, depth = [], 0, 0
    start = None
    while j < len(body):
        k = _skip_literal(body, j)
        if k != j:
            if start is None and not body.startswith("//", j) and not body.startswith("/*", j):
                start = j
            j = k
            continue
        c = body[j]
        if c == "#" and depth == 0 and (start is None or not body[start:j].strip()):
            e = body.find("\n", j)
            e = len(body) if e < 0 else e
            out.append((j, e))
            j, start = e, None
            continue
        if not c.isspace() and start is None:
            start = j
        if c in "({[":
            depth += 1
        elif c in ")}]":
            depth -= 1
            if depth == 0 and c == "}" and start is not None:
                # a block statement (if/for/while/{}) ends here unless ';' or 'else' follows
                rest = body[j + 1:].lstrip()
                if not rest.startswith(";") and not rest.startswith("else") and not re.match(r"while\b", rest):
                    out.append((start, j + 1))
                    start = None
        elif c == ";" and depth == 0:
            out.append((start, j + 1))
            start = None
        j += 1
    return out


DECL = re.compile(r"^\s*((?:(?:const|unsigned|signed|long|short|volatile)\s+)*"
                  r"(?:int|char|float|double|bool|size_t|u?int(?:8|16|32|64)_t|unsigned|long|short)\b[\s\*]*)(.*)$", re.S)


class Lowering:
    def __init__(self, src, mode):
        self.src, self.mode = src, mode
        self.funcs = find_functions(src)
        self.by_name = {f.name: f for f in self.funcs}
        self.entries = 0
        self.entry_structs = []
        self.entry_defs = []

    # -- task function body -------------------------------------------------
    def lower_function(self, f):
        params = {p.name for p in f.params}
        body = f.body
        # split at the top-level taskwaits
        segments, queues, last = [], [], 0
        for s, e in top_level_statements(body):
            pm = PRAGMA_AT.match(body, s)
            if pm and pm.group(1) == "taskwait":
                segments.append(body[last:s])
                queues.append(parse_queue(pm.group(2), f.line))
                last = e
        segments.append(body[last:])
        nested = [pm for pm in PRAGMA.finditer(body) if pm.group(1) == "taskwait"]
        if len(nested) != len(queues):
            raise LoweringError("line %d: a taskwait inside a nested block of '%s' is not supported"
                                % (f.line, f.name))
        # top-level declarations of each segment
        decls, seen = [], set(params)
        for i, seg in enumerate(segments):
            for s, e in top_level_statements(seg):
                st = seg[s:e]
                m = DECL.match(st)
                if not m or st.lstrip().startswith("#"):
                    continue
                base = " ".join(m.group(1).replace("*", " ").split())
                names = []
                for d in split_top(m.group(2).rstrip(";")):
                    dm = re.match(r"^(\**)\s*([A-Za-z_]\w*)\s*(\[.*)?(=.*)?$", d, re.S)
                    if not dm:
                        raise LoweringError("line %d: unsupported declaration '%s'" % (f.line, d))
                    if dm.group(2) in seen:
                        raise LoweringError("line %d: '%s' declared twice" % (f.line, dm.group(2)))
                    seen.add(dm.group(2))
                    names.append((dm.group(2), base + "*" * (m.group(1).count("*") + len(dm.group(1))),
                                  dm.group(3) is not None))
                decls.append((i, names))
        # a local lives in the frame when a later segment uses it, or when a
        # task's result is assigned to it (the result is read after the join)
        idents = [set(re.findall(r"[A-Za-z_]\w*", seg)) for seg in segments]
        lhs_names = set()
        for seg in segments:
            for pm in PRAGMA.finditer(seg):
                if pm.group(1) == "task":
                    st = seg[pm.end():statement_end(seg, pm.end())]
                    lm = re.match(r"^\s*([A-Za-z_]\w*)\s*=(?!=)", st)
                    if lm:
                        lhs_names.add(lm.group(1))
        hoisted = set(params)
        for i, names in decls:
            live = [n for n, _, _ in names if n in lhs_names or any(n in idents[k] for k in range(i + 1, len(segments)))]
            if live and len(live) != len(names):
                raise LoweringError("line %d: declare '%s' (used after a taskwait) in a declaration of its own"
                                    % (f.line, live[0]))
            for n, ctype, is_array in names:
                if n in live:
                    if is_array:
                        raise LoweringError("line %d: array '%s' cannot live across a taskwait" % (f.line, n))
                    hoisted.add(n)
                    f.locals.append(Param(ctype, n))
        segments = [replace_identifiers(seg, hoisted) for seg in segments]
        out_cases = []
        pending = []   # spawns with results joined at the next taskwait: (slot, lhs, callee)
        for i, seg in enumerate(segments):
            seg, spawned = self.lower_segment(f, seg, i)
            prologue = ""
            for slot, lhs, callee in pending:
                prologue += ("        if (__f->%s >= 0) {\n"
                             "            %s = ((%s*)__gtap_get_task_data(__f->%s))->__ret;\n"
                             "            %s__gtap_release_task_id(__f->%s);\n        }\n"
                             % (slot, lhs, self.by_name[callee].frame, slot,
                                "if (threadIdx.x == 0) " if self.mode == "block" else "", slot))
            pending = spawned
            if i < len(queues):
                q = queues[i] or "0"
                join = ("        if (__gtap_set_state_for_join_block(__tid, __ctx, %d, %s)) return;\n" % (i + 1, q)
                        if self.mode == "block" else
                        "        if (__gtap_set_state_for_join(__tid, __cc, %d, %s)) return;\n" % (i + 1, q))
            else:
                if pending:
                    raise LoweringError("line %d: the result of a task in '%s' is assigned but no taskwait follows"
                                        % (f.line, f.name))
                join = "        __gtap_finish_task(__tid, __ctx);\n        return;\n"
            out_cases.append("    case %d: {\n        int __cc = 0;\n        (void)__cc;\n%s%s\n%s    }\n"
                             % (i, prologue, seg, join))
        fields = ["    %s %s;" % (p.ctype, p.name) for p in f.params + f.locals]
        if f.ret != "void":
            fields.append("    %s __ret;" % f.ret)
        fields += ["    int %s;" % s for s in f.child_slots]
        if not fields:
            fields = ["    int __unused;"]
        frame = "struct %s {\n%s\n};\n" % (f.frame, "\n".join(fields))
        fn = ("__device__ void %s(void* __frame, int __tid, TaskContext* __ctx) {\n"
              "    %s* __f = (%s*)__frame;\n"
              "    (void)__f;\n"
              "    switch (__gtap_get_task_state(__tid)) {\n%s"
              "    default:\n        __gtap_finish_task(__tid, __ctx);\n        return;\n    }\n}\n"
              % (f.task, f.frame, f.frame, "".join(out_cases)))
        return frame, fn

    def lower_segment(self, f, seg, index):
        """Rewrite spawns, top-level declarations and returns of one segment."""
        spawned = []
        # spawns
        out, j = [], 0
        for pm in list(PRAGMA.finditer(seg)):
            if pm.group(1) in ("function", "entry"):
                raise LoweringError("line %d: '#pragma gtap %s' inside task function '%s'"
                                    % (f.line, pm.group(1), f.name))
            if pm.group(1) != "task":
                continue
            q = parse_queue(pm.group(2), f.line) or "0"
            s = pm.end()
            e = statement_end(seg, s)
            call = seg[s:e].strip()
            m = re.match(r"^(?:(?P<lhs>.+?)\s*=(?!=)\s*)?(?P<name>[A-Za-z_]\w*)\s*\((?P<args>.*)\)$", call, re.S)
            if not m or m.group("name") not in self.by_name:
                raise LoweringError("line %d: '#pragma gtap task' must precede a call to a task function, got '%s'"
                                    % (f.line, call))
            callee = self.by_name[m.group("name")]
            args = split_top(m.group("args"))
            if len(args) != len(callee.params):
                raise LoweringError("line %d: '%s' takes %d arguments" % (f.line, callee.name, len(callee.params)))
            before = seg[:pm.start()]
            lhs = m.group("lhs")
            if lhs and callee.ret == "void":
                raise LoweringError("line %d: '%s' returns nothing" % (f.line, callee.name))
            if lhs:
                if self._inside_loop(before):
                    raise LoweringError("line %d: a task whose result is assigned is inside a loop" % f.line)
                slot = "__child%d" % len(f.child_slots)
                f.child_slots.append(slot)
                spawned.append((slot, lhs, callee.name))
                tid_arg, retain = "&__f->" + slot, "true"
                # the slot is cleared when the segment starts
            else:
                tid_arg, retain = "nullptr", "false"
            assign = "".join("            __c->%s = %s;\n" % (p.name, a) for p, a in zip(callee.params, args))
            code = ("{\n            %s* __c = (%s*)__gtap_spawn_task(__ctx, __tid, &__cc, %s, %s, %s, %s);\n%s        }"
                    % (callee.frame, callee.frame, callee.task, q, tid_arg, retain, assign))
            out.append(seg[j:pm.start()])
            out.append(code)
            j = e + 1
        out.append(seg[j:])
        seg = "".join(out)
        clears = "".join("__f->%s = -1; " % s for s, _, _ in spawned)
        if clears:
            # block mode: ordered before any thread of the block spawns
            clears = ("        if (threadIdx.x == 0) { %s}\n        __syncthreads();\n" % clears if self.mode == "block"
                      else "        %s\n" % clears)
        # top-level declarations -> assignments
        stmts = top_level_statements(seg)
        out, j = [], 0
        for s, e in stmts:
            st = seg[s:e]
            m = DECL.match(st)
            if m and not st.lstrip().startswith("#") and "__f->" in m.group(2).split("=")[0]:
                # a hoisted declaration (all its names live in the frame)
                assigns = []
                for d in split_top(m.group(2).rstrip(";")):
                    dm = re.match(r"^(\**)\s*(__f->[A-Za-z_]\w*)\s*(=(.*))?$", d, re.S)
                    if dm and dm.group(3):
                        assigns.append("%s = %s;" % (dm.group(2), dm.group(4).strip()))
                out.append(seg[j:s])
                out.append(" ".join(assigns))
                j = e
        out.append(seg[j:])
        seg = "".join(out)
        # returns
        out, j = [], 0
        for m in re.finditer(r"\breturn\b", seg):
            if m.start() < j:
                continue
            e = statement_end(seg, m.end())
            expr = seg[m.end():e].strip()
            if expr:
                if f.ret == "void":
                    raise LoweringError("line %d: '%s' returns void" % (f.line, f.name))
                code = "{ __f->__ret = (%s); __gtap_finish_task(__tid, __ctx); return; }" % expr
            else:
                code = "{ __gtap_finish_task(__tid, __ctx); return; }"
            out.append(seg[j:m.start()])
            out.append(code)
            j = e + 1
        out.append(seg[j:])
        return clears + "".join(out), spawned

    @staticmethod
    def _loop_header(head):
        # head: the text before a '{' or a braceless statement; True if it ends a loop header
        head = head.rstrip()
        if re.search(r"\bdo$", head):
            return True
        if not head.endswith(")"):
            return False
        depth, k = 0, len(head) - 1
        while k >= 0:
            if head[k] == ")":
                depth += 1
            elif head[k] == "(":
                depth -= 1
                if depth == 0:
                    break
            k -= 1
        return re.search(r"\b(for|while)\s*$", head[:max(k, 0)]) is not None

    @classmethod
    def _inside_loop(cls, before):
        # any enclosing block, or the braceless statement itself, is a loop body
        if cls._loop_header(before):
            return True
        depth, k = 0, len(before) - 1
        while k >= 0:
            if before[k] == "}":
                depth += 1
            elif before[k] == "{":
                if depth == 0:
                    if cls._loop_header(before[:k]):
                        return True
                else:
                    depth -= 1
            k -= 1
        return False

    # -- entries ----------------------------------------------------------
    def lower_entry(self, text_after, line):
        e = statement_end(text_after, 0)
        call = text_after[:e].strip()
        m = re.match(r"^(?:(?P<lhs>.+?)\s*=(?!=)\s*)?(?P<name>[A-Za-z_]\w*)\s*\((?P<args>.*)\)$", call, re.S)
        if not m or m.group("name") not in self.by_name:
            raise LoweringError("line %d: '#pragma gtap entry' must precede a call to a task function" % line)
        g = self.by_name[m.group("name")]
        args = split_top(m.group("args"))
        if len(args) != len(g.params):
            raise LoweringError("line %d: '%s' takes %d arguments" % (line, g.name, len(g.params)))
        k = self.entries
        self.entries += 1
        lhs = m.group("lhs")
        if not lhs:
            # the root task itself is task 0
            fill = "".join("        __e->%s = %s;\n" % (p.name, a) for p, a in zip(g.params, args))
            code = ("if (blockIdx.x == 0 && threadIdx.x == 0) {\n"
                    "        __gtap_push_initial_task(%s, 0);\n"
                    "        %s* __e = (%s*)__gtap_get_task_data(0);\n%s    }\n"
                    "    __gtap_execute_task_loop_device();" % (g.task, g.frame, g.frame, fill))
            return code, e + 1
        if g.ret == "void":
            raise LoweringError("line %d: '%s' returns nothing" % (line, g.name))
        ef = "__gtap_entry_frame%d" % k
        fields = "".join("    %s a%d;\n" % (p.ctype, i) for i, p in enumerate(g.params)) + "    int __child;\n"
        fill = "".join("        __e->a%d = %s;\n" % (i, a) for i, a in enumerate(args))
        assign = "".join("            __c->%s = __f->a%d;\n" % (p.name, i) for i, p in enumerate(g.params))
        once = "if (threadIdx.x == 0) " if self.mode == "block" else ""
        join = ("__gtap_set_state_for_join_block(__tid, __ctx, 1, 0)" if self.mode == "block"
                else "__gtap_set_state_for_join(__tid, __cc, 1, 0)")
        self.entry_structs.append("struct %s {\n%s};\n"
                                  "__device__ void __gtap_entry%d(void* __frame, int __tid, TaskContext* __ctx);\n"
                                  % (ef, fields, k))
        self.entry_defs.append(
            "__device__ void __gtap_entry%d(void* __frame, int __tid, TaskContext* __ctx) {\n"
            "    %s* __f = (%s*)__frame;\n"
            "    switch (__gtap_get_task_state(__tid)) {\n"
            "    case 0: {\n        int __cc = 0;\n        (void)__cc;\n"
            "        %s{\n            %s* __c = (%s*)__gtap_spawn_task(__ctx, __tid, &__cc, %s, 0, &__f->__child, true);\n"
            "%s        }\n"
            "        if (%s) return;\n    }\n"
            "    case 1: {\n"
            "        %s{\n            %s = ((%s*)__gtap_get_task_data(__f->__child))->__ret;\n"
            "            __gtap_release_task_id(__f->__child);\n        }\n"
            "        __gtap_finish_task(__tid, __ctx);\n        return;\n    }\n"
            "    default:\n        __gtap_finish_task(__tid, __ctx);\n        return;\n    }\n}\n"
            % (k, ef, ef, once, g.frame, g.frame, g.task, assign, join, once, lhs, g.frame))
        code = ("if (blockIdx.x == 0 && threadIdx.x == 0) {\n"
                "        __gtap_push_initial_task(__gtap_entry%d, 0);\n"
                "        %s* __e = (%s*)__gtap_get_task_data(0);\n%s    }\n"
                "    __gtap_execute_task_loop_device();" % (k, ef, ef, fill))
        return code, e + 1

    # -- whole file ------------------------------------------------------------
    def run(self):
        if not self.funcs:
            raise LoweringError("no '#pragma gtap function' in the input")
        src = self.src
        frames, bodies = [], []
        for f in self.funcs:
            fr, fn = self.lower_function(f)
            frames.append(fr)
            bodies.append(fn)
        # entries, outside the task functions
        out, j = [], 0
        for pm in PRAGMA.finditer(src):
            if pm.group(1) != "entry":
                continue
            if any(f.start <= pm.start() < f.end for f in self.funcs):
                continue
            code, used = self.lower_entry(src[pm.end():], line_of(src, pm.start()))
            out.append(src[j:pm.start()])
            out.append(code)
            j = pm.end() + used
        out.append(src[j:])
        src = "".join(out)
        # drop the original task functions; declarations go where the first one was
        funcs = find_functions(src)
        first = funcs[0].start
        decls = ("// ---- lowered by gtap_b200.lower ----\n" + "".join(frames)
                 + "".join("__device__ void %s(void* __frame, int __tid, TaskContext* __ctx);\n" % f.task
                           for f in self.funcs) + "".join(self.entry_structs))
        sizes = [f.frame for f in self.funcs] + ["__gtap_entry_frame%d" % k for k in range(len(self.entry_defs))]
        size_expr = "sizeof(%s)" % sizes[0]
        for s in sizes[1:]:
            size_expr = "(sizeof(%s) > %s ? sizeof(%s) : %s)" % (s, size_expr, s, size_expr)
        # entry tasks and the frame size follow the last task function
        tail = "".join(self.entry_defs) + "const size_t __gtap_auto_task_data_size = %s;\n" % size_expr
        pieces, j = [], 0
        for k, f in enumerate(funcs):
            pieces.append(src[j:f.start])
            if k == 0:
                pieces.append(decls)
            pieces.append(bodies[k])
            if k == len(funcs) - 1:
                pieces.append(tail)
            j = f.end
        pieces.append(src[j:])
        return "".join(pieces)


def lower_source(src, mode=None):
    """Lowered text of a pragma program; mode 'thread' or 'block' (default:
    from the gtap header it includes)."""
    if mode is None:
        mode = "block" if re.search(r'#\s*include\s*[<"]gtap_block\.cuh[>"]', src) else "thread"
    if mode not in ("thread", "block"):
        raise LoweringError("mode must be 'thread' or 'block'")
    return Lowering(src, mode).run()


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("input")
    ap.add_argument("-o", "--output", required=True)
    ap.add_argument("--mode", choices=["thread", "block"], default=None)
    a = ap.parse_args(argv)
    try:
        with open(a.input) as f:
            out = lower_source(f.read(), a.mode)
    except LoweringError as e:
        sys.stderr.write("%s: %s\n" % (a.input, e))
        return 1
    with open(a.output, "w") as f:
        f.write(out)
    return 0


if __name__ == "__main__":
    sys.exit(main())
