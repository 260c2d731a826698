"""Source-to-source lowering of `#pragma gtap` programs to the task ABI.

The reference's compiler front end (clang-gtap) is not part of its checkout,
so programs written with the pragmas of examples/README.md:70-79 cannot be
built from it.  This module lowers the same pragmas, for a restricted subset
of C++, into the switch state machines the task ABI expects
(include/gtap_thread.cuh, include/gtap_block.cuh), which nvcc then compiles:

    python -m gtap_b200.lower prog.cu -o prog_lowered.cu [--mode thread|block] [--results retain|parent]

Pragmas
  #pragma gtap function               before a `__device__ T name(params) {...}`
  #pragma gtap task [queue(expr)]     before `name(args);` or `lhs = name(args);`
  #pragma gtap taskwait [queue(expr)] waits for the children spawned since the last one
  #pragma gtap entry                  in a __global__ kernel, before `[lhs =] name(args);`

Lowering (the contract of the reference's task ABI):
  * each task function becomes `void name__gtap_task(void*, int, TaskContext*)`
    with a frame struct `__gtap_frame_name` holding its parameters, the
    locals that live across a taskwait, the return value (`__ret`) and one
    child id per spawn site whose result is used;
  * the body becomes one switch on __gtap_get_task_state; a taskwait becomes
    __gtap_set_state_for_join (thread mode) or __gtap_set_state_for_join_block
    (block mode), returning while children are outstanding, followed by the
    case label the task resumes at -- inside the if/else branch that holds
    the taskwait, if it is nested;
  * a local in scope at a resume point moves to the frame when it is used
    after that point or assigned a task's result; otherwise its initialiser
    is split from its declaration, so no jump to a label crosses one;
  * a spawn becomes __gtap_spawn_task with the arguments written into the
    child's frame; a child whose result is assigned is retained, and its
    result is read from its frame, and its id released, right after the
    taskwait that joins it (the left-hand side is evaluated there); a local
    that only receives results of unconditional spawns joined at one
    taskwait, and is read only before the next one, stays a plain local;
  * `return e;` stores e in the frame and calls __gtap_finish_task;
  * an entry pushes the root as task 0 (through a small entry task when its
    result is assigned) and runs __gtap_execute_task_loop_device;
  * the output starts with `#define GTAP_DIRECT_DISPATCH 1` and defines
    __gtap_dispatch, which the drop-in headers call to run a task: the stored
    function pointer is compared with each task function and the match is
    called directly, so the bodies are inlined into the worker loop.

Restrictions (reported as LoweringError with the source line):
  * no taskwait inside a loop or a switch, or as the body of an if/else
    without braces; in block mode every thread of the block reaches it;
  * locals that live across a taskwait have builtin arithmetic or pointer
    types, are not arrays, and have a name no other local of the function
    uses; no local shadows a parameter;
  * a spawn whose result is assigned is not inside a loop, and the next
    taskwait after it is in its own block or an enclosing one;
  * task functions are only called through `#pragma gtap task` / `entry`;
  * a result is assigned with `=`, not a compound assignment.

--results parent (thread mode, experimental): instead of retained child
frames, a child with a result writes it into its parent's frame (through a
4-byte destination word in its own frame) before it finishes, and every task
reads its frame from the words the worker loads with the task header
(GTAP_FRAME_WORDS, __gtap_dispatch_words), working on a copy that is written
back before a join.  Results then go to plain locals or parameters of the
callee's return type, one per local and join, with no return between a spawn
and its join.  In thread mode the entry kernel gets launch bounds that keep
every worker resident (both result schemes).
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
    def __init__(self, name, ret, params, body, start, end, line, body_line=None):
        self.name, self.ret, self.params, self.body = name, ret, params, body
        self.start, self.end, self.line = start, end, line
        self.body_line = line if body_line is None else body_line   # source line of the body's first character
        self.locals = []        # [Param]
        self.child_slots = []   # names of child-id fields
        self.cond_slots = []    # those whose spawn may not run before its join

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
                                  m.start(), bc + 1, line_of(src, m.start()), line_of(src, bo + 1)))
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


GENERIC_DECL = re.compile(r"^\s*(?:(?:const|volatile|struct|static)\s+)*([A-Za-z_][\w:]*(?:\s*<[^;{}]*>)?)"
                          r"[\s\*&]+([A-Za-z_]\w*)\s*(?:=|;|\[|,|\(|\{)")
NOT_TYPES = {"return", "goto", "delete", "throw", "case", "else", "do", "typedef", "using", "break",
             "continue", "new", "sizeof", "if", "for", "while", "switch", "asm"}
CALL = re.compile(r"^(?:(?P<lhs>.+?)\s*=(?!=)\s*)?(?P<name>[A-Za-z_]\w*)\s*\((?P<args>.*)\)$", re.S)


def _blocks(body):
    """(open, close) of every brace pair in body (literals and comments skipped)."""
    out, stack, j = [], [], 0
    while j < len(body):
        k = _skip_literal(body, j)
        if k != j:
            j = k
            continue
        if body[j] == "{":
            stack.append(j)
        elif body[j] == "}":
            if not stack:
                raise LoweringError("unbalanced '}' at line %d of a task function" % line_of(body, j))
            out.append((stack.pop(), j))
        j += 1
    if stack:
        raise LoweringError("unbalanced '{' at line %d of a task function" % line_of(body, stack[-1]))
    return out


def _header_kind(head):
    """The control keyword whose header ends `head` (the text before a '{' or a
    braceless statement): 'for', 'while', 'do', 'if', 'else', 'switch' or None."""
    head = head.rstrip()
    m = re.search(r"\b(do|else)$", head)
    if m:
        return m.group(1)
    if not head.endswith(")"):
        return None
    depth, k = 0, len(head) - 1
    while k >= 0:
        if head[k] == ")":
            depth += 1
        elif head[k] == "(":
            depth -= 1
            if depth == 0:
                break
        k -= 1
    m = re.search(r"\b(for|while|if|switch)\s*$", head[:max(k, 0)])
    return m.group(1) if m else None


def _declarators(m, line):
    """[(name, stars, dims, init)] of a DECL match."""
    out = []
    for d in split_top(m.group(2).rstrip().rstrip(";")):
        dm = re.match(r"^(\**)\s*([A-Za-z_]\w*)\s*((?:\[[^\]]*\]\s*)*)(?:=(.*))?$", d, re.S)
        if not dm:
            raise LoweringError("line %d: unsupported declaration '%s'" % (line, d))
        out.append((dm.group(2), m.group(1).count("*") + len(dm.group(1)), dm.group(3).strip(),
                    dm.group(4).strip() if dm.group(4) is not None else None))
    return out


def _words(text, word):
    """Matches of the identifier `word` outside string/char literals and comments."""
    out, j = [], 0
    ident = re.compile(r"[A-Za-z_]\w*")
    while j < len(text):
        k = _skip_literal(text, j)
        if k != j:
            j = k
            continue
        m = ident.match(text, j)
        if not m:
            j += 1
            continue
        if m.group(0) == word:
            out.append(m)
        j = m.end()
    return out


def _is_written(text, name):
    """True if `name` (not as a member) is assigned, incremented or has its
    address taken anywhere in text."""
    j = 0
    ident = re.compile(r"[A-Za-z_]\w*")
    while j < len(text):
        k = _skip_literal(text, j)
        if k != j:
            j = k
            continue
        m = ident.match(text, j)
        if not m:
            j += 1
            continue
        if m.group(0) == name:
            before = text[:m.start()].rstrip()
            after = text[m.end():]
            if not (before.endswith(".") or before.endswith("->")):
                if re.match(r"\s*(?:<<|>>|[-+*/%&|^])?=(?!=)", after) or re.match(r"\s*(?:\+\+|--)", after):
                    return True
                if re.search(r"(?:\+\+|--)$", before) or (before.endswith("&") and not before.endswith("&&")):
                    return True
        j = m.end()
    return False


def _local_type(m, stars):
    """Type of a declarator: the declaration's base type plus its stars; a
    top-level const is dropped (the variable is assigned after its declaration)."""
    words = m.group(1).replace("*", " ").split()
    if stars == 0:
        words = [w for w in words if w != "const"]
    return " ".join(words) + "*" * stars


class Lowering:
    def __init__(self, src, mode, results="retain"):
        self.src, self.mode, self.results = src, mode, results
        self.parent = results == "parent"
        if self.parent and mode != "thread":
            raise LoweringError("--results parent needs thread mode")
        self.funcs = find_functions(src)
        self.by_name = {f.name: f for f in self.funcs}
        self.entries = 0
        self.entry_structs = []
        self.entry_defs = []

    # -- task function body -------------------------------------------------
    def lower_function(self, f):
        """One switch on the task state; each taskwait becomes a join that
        returns while children are outstanding, followed by the case label the
        task resumes at.  A taskwait may sit in nested if/else blocks, not in
        a loop or a switch.  Locals in scope at a resume point either move to
        the frame (when used after it, or assigned a task's result) or have
        their initialiser split off, so no jump crosses an initialisation."""
        body = f.body
        params = {p.name for p in f.params}
        blocks = _blocks(body)
        whole = (-1, len(body))

        def chain(pos):
            return {b for b in blocks if b[0] < pos < b[1]}

        def ln(pos):
            # source line of a position in the original body
            return f.body_line + body.count("\n", 0, pos)

        prags = list(PRAGMA.finditer(body))
        for pm in prags:
            if pm.group(1) in ("function", "entry"):
                raise LoweringError("line %d: '#pragma gtap %s' inside task function '%s'"
                                    % (ln(pm.start()), pm.group(1), f.name))
            if pm.group(1) not in ("task", "taskwait"):
                raise LoweringError("line %d: unknown pragma '#pragma gtap %s'" % (ln(pm.start()), pm.group(1)))
        waits = [pm for pm in prags if pm.group(1) == "taskwait"]
        tasks = [pm for pm in prags if pm.group(1) == "task"]
        for pm in waits:
            before = body[:pm.start()]
            if self._inside_loop(before):
                raise LoweringError("line %d: a taskwait inside a loop of '%s' is not supported" % (ln(pm.start()), f.name))
            if _header_kind(before) is not None:
                raise LoweringError("line %d: a taskwait in '%s' is the body of an if/else without braces"
                                    % (ln(pm.start()), f.name))
            for o, _ in chain(pm.start()):
                if _header_kind(body[:o]) == "switch":
                    raise LoweringError("line %d: a taskwait inside a switch of '%s' is not supported"
                                        % (ln(pm.start()), f.name))
        # spawns whose result is assigned, and the taskwait that joins each
        joins, cond, lhs_idents = {}, {}, set()
        bare = {}       # bare identifier on the left -> [(task index, start, end of the spawn statement)]
        for ti, pm in enumerate(tasks):
            call = body[pm.end():statement_end(body, pm.end())].strip()
            m = CALL.match(call)
            if not m or not m.group("lhs"):
                continue
            if re.search(r"[-+*/%&|^<>!]$", m.group("lhs").strip()):
                raise LoweringError("line %d: a task's result can only be assigned with '=', not '%s='"
                                    % (ln(pm.start()), m.group("lhs").strip().split()[-1][-1]))
            if self._inside_loop(body[:pm.start()]):
                raise LoweringError("line %d: a task whose result is assigned is inside a loop" % ln(pm.start()))
            nxt = next((k for k, w in enumerate(waits) if w.start() > pm.start()), None)
            if nxt is None:
                raise LoweringError("line %d: the result of a task in '%s' is assigned but no taskwait follows"
                                    % (ln(pm.start()), f.name))
            if not chain(waits[nxt].start()) <= chain(pm.start()):
                raise LoweringError("line %d: the result of a task in '%s' is joined only inside a nested block"
                                    % (ln(pm.start()), f.name))
            joins[ti] = nxt
            # conditional: the spawn sits in a block the taskwait is not in
            cond[ti] = chain(waits[nxt].start()) != chain(pm.start())
            lhs_idents |= set(re.findall(r"[A-Za-z_]\w*", m.group("lhs")))
            if re.match(r"^[A-Za-z_]\w*$", m.group("lhs").strip()):
                bare.setdefault(m.group("lhs").strip(), []).append((ti, pm.start(), statement_end(body, pm.end())))
        if self.parent:
            self._check_parent_results(f, body, tasks, waits, joins, bare, ln)
        # declarations at the top level of every block
        decls = []      # (start, end, block, match or None, [(name, stars, dims, init)])
        for o, c in blocks + [whole]:
            for s, e in top_level_statements(body[o + 1:c]):
                s, e = s + o + 1, e + o + 1
                st = body[s:e]
                if st.lstrip().startswith("#"):
                    continue
                m = DECL.match(st)
                if m:
                    decls.append((s, e, (o, c), m, _declarators(m, ln(s))))
                    continue
                g = GENERIC_DECL.match(st)
                if g and g.group(1) not in NOT_TYPES:
                    decls.append((s, e, (o, c), None, [(g.group(2), 0, "", None)]))
        # result-only locals: assigned the results of unconditional spawns
        # joined at one taskwait and read only between that taskwait and the
        # next.  The join always overwrites them, so they stay plain locals
        # and the frame stays small.
        result_only = set()
        for name, sites in ([] if self.parent else bare.items()):
            ks = {joins[ti] for ti, _, _ in sites}
            if len(ks) != 1 or any(cond[ti] for ti, _, _ in sites) or name in params:
                continue
            k = ks.pop()
            mine = [d for d in decls if any(n == name for n, _, _, _ in d[4])]
            if len(mine) != 1 or mine[0][3] is None:
                continue
            ds, de, (o, c), _, names = mine[0]
            if any(n == name and dims for n, _, dims, _ in names) or not (o < waits[k].start() < c):
                continue
            lo = waits[k].end()
            hi = waits[k + 1].start() if k + 1 < len(waits) else len(body)
            ok = True
            for um in re.finditer(r"\b%s\b" % re.escape(name), body):
                u = um.start()
                if ds <= u < de or any(a <= u <= b for _, a, b in sites) or lo <= u < hi:
                    continue
                ok = False
                break
            if ok:
                result_only.add(name)
        hoist, count = {}, {}
        for s, e, (o, c), m, names in decls:
            crossing = [w for w in waits if e <= w.start() < c]
            after = set()
            for w in crossing:
                after |= set(re.findall(r"[A-Za-z_]\w*", body[w.start():c]))
            for name, stars, dims, init in names:
                count[name] = count.get(name, 0) + 1
                if name in params:
                    raise LoweringError("line %d: local '%s' shadows a parameter of '%s'" % (ln(s), name, f.name))
                if m is None:
                    if crossing:
                        raise LoweringError("line %d: local '%s' of '%s' has a type the lowering cannot keep "
                                            "across a taskwait; declare it after the taskwait or in a block "
                                            "that ends before it" % (ln(s), name, f.name))
                    continue
                if name not in result_only and (name in lhs_idents or (crossing and name in after)):
                    if dims:
                        raise LoweringError("line %d: array '%s' cannot live across a taskwait" % (ln(s), name))
                    hoist[name] = _local_type(m, stars)
        for name in hoist:
            if count[name] > 1:
                raise LoweringError("line %d: '%s' is declared twice in '%s'; a local that lives across a "
                                    "taskwait needs a name of its own" % (f.line, name, f.name))
        if self.parent:
            types = dict(hoist)
            types.update({p.name: " ".join(p.ctype.split()) for p in f.params})
            for name, sites in bare.items():
                for ti, a, _ in sites:
                    callee = self.by_name[CALL.match(body[tasks[ti].end():statement_end(body, tasks[ti].end())]
                                                     .strip()).group("name")]
                    if types.get(name) != callee.ret:
                        raise LoweringError("line %d: with --results parent, '%s' must be a local or parameter of "
                                            "type '%s' (the return type of '%s')" % (ln(a), name, callee.ret,
                                                                                     callee.name))
            f.targets = sorted(set(bare))
        # rewrite the declarations in scope at a resume point
        edits = []
        for s, e, (o, c), m, names in decls:
            if m is None or not (any(e <= w.start() < c for w in waits) or any(n in hoist for n, _, _, _ in names)):
                continue
            parts = []
            for name, stars, dims, init in names:
                if name in hoist:
                    if init is not None:
                        parts.append("%s = %s;" % (name, init))
                    continue
                if dims and init is not None:
                    raise LoweringError("line %d: array '%s' with an initialiser is in scope at a taskwait; "
                                        "declare it after the taskwait" % (f.line, name))
                parts.append("%s %s%s;" % (_local_type(m, stars), name, dims))
                if init is not None:
                    parts.append("%s = %s;" % (name, init))
            edits.append((s, e, " ".join(parts)))
        out, j = [], 0
        for s, e, text in sorted(edits):
            out.append(body[j:s])
            out.append(text)
            j = e
        out.append(body[j:])
        # parameters the body never writes are read from the frame once, on entry
        readonly = [p for p in f.params if not _is_written(f.body, p.name)]
        body = replace_identifiers("".join(out), (params - {p.name for p in readonly}) | set(hoist))
        for n in hoist:
            f.locals.append(Param(hoist[n], n))
        body, at_wait = self.lower_spawns(f, body, joins, cond)
        body = self.lower_returns(f, body)
        # with --results parent the task works on a copy of its frame: write
        # it back before a join that may suspend it
        writeback = "*__fm = *__f; " if self.parent else ""
        # taskwaits -> join + resume label + results of the joined children
        out, j, k = [], 0, 0
        for pm in PRAGMA.finditer(body):
            if pm.group(1) != "taskwait":
                continue
            q = parse_queue(pm.group(2), f.line) or "0"
            join = ("if (__gtap_set_state_for_join_block(__tid, __ctx, %d, %s)) return;" % (k + 1, q)
                    if self.mode == "block" else
                    "%sif (__gtap_set_state_for_join(__tid, __cc, %d, %s)) return;" % (writeback, k + 1, q))
            # every result is read before any id is released, so the reads
            # overlap; an unconditional spawn always ran before this join
            reads, releases = "", ""
            for slot, lhs, callee, conditional in at_wait.get(k, []):
                guard = "if (__f->%s >= 0) " % slot if conditional else ""
                reads += ("        %s%s = ((%s*)__gtap_get_task_data(__f->%s))->__ret;\n"
                          % (guard, lhs, self.by_name[callee].frame, slot))
                releases += ("        %s%s__gtap_release_task_id(__f->%s);\n"
                             % (guard, "if (threadIdx.x == 0) " if self.mode == "block" else "", slot))
            results = reads + releases
            out.append(body[j:body.index("#", pm.start())])
            out.append("%s\n    case %d:\n        __cc = 0;\n%s" % (join, k + 1, results))
            j = pm.end()
            k += 1
        out.append(body[j:])
        body = "".join(out)
        clears = "".join("__f->%s = -1; " % s for s in f.cond_slots)
        if clears:
            # block mode: ordered before any thread of the block spawns
            clears = ("        if (threadIdx.x == 0) { %s}\n        __syncthreads();\n" % clears if self.mode == "block"
                      else "        %s\n" % clears)
        fields = ["    %s %s;" % (p.ctype, p.name) for p in f.params + f.locals]
        if f.ret != "void":
            # parent mode: where the result goes (0: nowhere), else the result itself
            fields.append("    unsigned __dst;" if self.parent else "    %s __ret;" % f.ret)
        fields += ["    int %s;" % s for s in f.child_slots]
        if not fields:
            fields = ["    int __unused;"]
        frame = "struct %s {\n%s\n};\n" % (f.frame, "\n".join(fields))
        if self.parent:
            frame += "".join("static_assert(offsetof(%s, %s) %% 4 == 0 && offsetof(%s, %s) < 128, "
                             "\"a task result is delivered into the first 128 bytes of the frame\");\n"
                             % (f.frame, t, f.frame, t) for t in getattr(f, "targets", []))
            return frame, self._parent_function(f, readonly, body)
        fn = ("__device__ void %s(void* __frame, int __tid, TaskContext* __ctx) {\n"
              "    %s* __f = (%s*)__frame;\n"
              "    (void)__f;\n"
              "%s"
              "    int __cc = 0;\n"
              "    (void)__cc;\n"
              "    switch (__gtap_get_task_state(__tid)) {\n"
              "    case 0: {\n%s%s\n    }\n"
              "        __gtap_finish_task(__tid, __ctx);\n        return;\n"
              "    default:\n        __gtap_finish_task(__tid, __ctx);\n        return;\n    }\n}\n"
              % (f.task, f.frame, f.frame,
                 "".join("    %s %s = __f->%s;\n    (void)%s;\n" % (p.ctype, p.name, p.name, p.name) for p in readonly),
                 clears, body))
        return frame, fn

    def lower_spawns(self, f, body, joins, cond):
        """`#pragma gtap task [queue(q)]` + call -> __gtap_spawn_task with the
        arguments written into the child's frame.  Returns the text and, per
        taskwait index, the (slot, lhs, callee) of the results it joins."""
        at_wait = {}
        out, j, ti = [], 0, 0
        for pm in list(PRAGMA.finditer(body)):
            if pm.group(1) != "task":
                continue
            q = parse_queue(pm.group(2), f.line) or "0"
            s = pm.end()
            e = statement_end(body, s)
            call = body[s:e].strip()
            m = CALL.match(call)
            if not m or m.group("name") not in self.by_name:
                raise LoweringError("line %d: '#pragma gtap task' must precede a call to a task function, got '%s'"
                                    % (f.line, call))
            callee = self.by_name[m.group("name")]
            args = split_top(m.group("args"))
            if len(args) != len(callee.params):
                raise LoweringError("line %d: '%s' takes %d arguments" % (f.line, callee.name, len(callee.params)))
            lhs = m.group("lhs")
            if lhs and callee.ret == "void":
                raise LoweringError("line %d: '%s' returns nothing" % (f.line, callee.name))
            if self.parent:
                assign = "".join("        __c->%s = %s;\n" % (p.name, a) for p, a in zip(callee.params, args))
                if callee.ret != "void":
                    field = lhs.strip()[len("__f->"):] if lhs else None
                    assign += ("        __c->__dst = __gtap_dst(__tid, offsetof(%s, %s));\n" % (f.frame, field)
                               if lhs else "        __c->__dst = 0u;\n")
                code = ("{\n        %s* __c = (%s*)__gtap_spawn_task(__ctx, __tid, &__cc, %s, %s, nullptr, false);\n%s    }"
                        % (callee.frame, callee.frame, callee.task, q, assign))
                out.append(body[j:body.index("#", pm.start())])
                out.append(code)
                j = e + 1
                ti += 1
                continue
            if lhs:
                slot = "__child%d" % len(f.child_slots)
                f.child_slots.append(slot)
                at_wait.setdefault(joins[ti], []).append((slot, lhs.strip(), callee.name, cond[ti]))
                if cond[ti]:
                    f.cond_slots.append(slot)   # cleared on entry: the spawn may not run
                tid_arg, retain = "&__f->" + slot, "true"
            else:
                tid_arg, retain = "nullptr", "false"
            assign = "".join("        __c->%s = %s;\n" % (p.name, a) for p, a in zip(callee.params, args))
            code = ("{\n        %s* __c = (%s*)__gtap_spawn_task(__ctx, __tid, &__cc, %s, %s, %s, %s);\n%s    }"
                    % (callee.frame, callee.frame, callee.task, q, tid_arg, retain, assign))
            out.append(body[j:body.index("#", pm.start())])
            out.append(code)
            j = e + 1
            ti += 1
        out.append(body[j:])
        return "".join(out), at_wait

    def lower_returns(self, f, body):
        """`return e;` -> the result into the frame, then __gtap_finish_task."""
        out, j = [], 0
        for m in _words(body, "return"):
            if m.start() < j:
                continue
            e = statement_end(body, m.end())
            expr = body[m.end():e].strip()
            if expr:
                if f.ret == "void":
                    raise LoweringError("line %d: '%s' returns void" % (f.line, f.name))
                code = ("{ if (__f->__dst) __gtap_deliver<%s>(__f->__dst, (%s)); __gtap_finish_task(__tid, __ctx); return; }"
                        % (f.ret, expr) if self.parent else
                        "{ __f->__ret = (%s); __gtap_finish_task(__tid, __ctx); return; }" % expr)
            else:
                code = "{ __gtap_finish_task(__tid, __ctx); return; }"
            out.append(body[j:m.start()])
            out.append(code)
            j = e + 1
        out.append(body[j:])
        return "".join(out)

    def _check_parent_results(self, f, body, tasks, waits, joins, bare, ln):
        """--results parent: every result goes to a plain local or parameter,
        one spawn per local and join, and no return may come between a spawn
        and the taskwait that joins it (the child writes into this frame)."""
        for ti, pm in enumerate(tasks):
            m = CALL.match(body[pm.end():statement_end(body, pm.end())].strip())
            if not m or not m.group("lhs"):
                continue
            if not re.match(r"^[A-Za-z_]\w*$", m.group("lhs").strip()):
                raise LoweringError("line %d: with --results parent, a task's result must be assigned to a plain "
                                    "local or parameter, not '%s'" % (ln(pm.start()), m.group("lhs").strip()))
            w = waits[joins[ti]]
            if _words(body[pm.end():w.start()], "return"):
                raise LoweringError("line %d: with --results parent, no return may come between a spawn whose "
                                    "result is assigned and its taskwait" % ln(pm.start()))
        for name, sites in bare.items():
            ks = [joins[ti] for ti, _, _ in sites]
            if len(ks) != len(set(ks)):
                raise LoweringError("line %d: with --results parent, '%s' receives two results at one taskwait"
                                    % (ln(sites[0][1]), name))

    def _parent_function(self, f, readonly, body):
        """Task text for --results parent: a copy of the frame, loaded from the
        words the worker read with the header, and the ABI entry point."""
        return ("__device__ __forceinline__ void %s__gtap_run(void* __frame, int __tid, TaskContext* __ctx, "
                "const int4& __w0, const int4& __w1, bool __words) {\n"
                "    %s* __fm = (%s*)__frame;\n"
                "    %s __fl;\n"
                "    __gtap_load_frame(&__fl, __fm, __w0, __w1, __words);\n"
                "    %s* __f = &__fl;\n"
                "%s"
                "    int __cc = 0;\n"
                "    (void)__cc;\n"
                "    switch (__gtap_get_task_state(__tid)) {\n"
                "    case 0: {\n%s\n    }\n"
                "        __gtap_finish_task(__tid, __ctx);\n        return;\n"
                "    default:\n        __gtap_finish_task(__tid, __ctx);\n        return;\n    }\n}\n"
                "__device__ void %s(void* __frame, int __tid, TaskContext* __ctx) {\n"
                "    const int4 __z = make_int4(0, 0, 0, 0);\n"
                "    %s__gtap_run(__frame, __tid, __ctx, __z, __z, false);\n}\n"
                % (f.name, f.frame, f.frame, f.frame, f.frame,
                   "".join("    %s %s = __f->%s;\n    (void)%s;\n" % (p.ctype, p.name, p.name, p.name) for p in readonly),
                   body, f.task, f.name))

    @staticmethod
    def _loop_header(head):
        # head: the text before a '{' or a braceless statement; True if it ends a loop header
        return _header_kind(head) in ("for", "while", "do")

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
            if self.parent and g.ret != "void":
                fill += "        __e->__dst = 0u;\n"
            code = ("if (blockIdx.x == 0 && threadIdx.x == 0) {\n"
                    "        __gtap_push_initial_task(%s, 0);\n"
                    "        %s* __e = (%s*)__gtap_get_task_data(0);\n%s    }\n"
                    "    __gtap_execute_task_loop_device();" % (g.task, g.frame, g.frame, fill))
            return code, e + 1
        if g.ret == "void":
            raise LoweringError("line %d: '%s' returns nothing" % (line, g.name))
        ef = "__gtap_entry_frame%d" % k
        if self.parent:
            return self._parent_entry(g, args, lhs, k, e)
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

    @staticmethod
    def _bound_kernel(head):
        """Thread mode: give the kernel that holds the entry launch bounds
        asking for every worker block to be resident (GTAP_GRID_SIZE blocks
        over 148 SMs, at most 32 blocks and 2048 threads per SM).  A persistent
        worker that is not resident only starts when a resident one exits, so
        without the bounds a register-heavy program ran with fewer workers
        than it launched; with --results parent the bounds also keep the
        preloaded frame words from raising the register count."""
        m = None
        for m in re.finditer(r"__global__\s+void\s+", head):
            pass
        if m is None or "__launch_bounds__" in head[m.start():]:
            return head
        per_sm = "((GTAP_GRID_SIZE + 147) / 148)"
        cap = "(2048 / GTAP_BLOCK_SIZE < 32 ? 2048 / GTAP_BLOCK_SIZE : 32)"
        bounds = "__launch_bounds__(GTAP_BLOCK_SIZE, (%s < %s ? %s : %s)) " % (per_sm, cap, per_sm, cap)
        return head[:m.end()] + bounds + head[m.end():]

    def _parent_entry(self, g, args, lhs, k, e):
        """Entry whose result is assigned, --results parent: the root delivers
        its result into the entry task's frame."""
        ef = "__gtap_entry_frame%d" % k
        fields = "".join("    %s a%d;\n" % (p.ctype, i) for i, p in enumerate(g.params)) + "    %s __res;\n" % g.ret
        fill = "".join("        __e->a%d = %s;\n" % (i, a) for i, a in enumerate(args))
        assign = "".join("            __c->%s = __f->a%d;\n" % (p.name, i) for i, p in enumerate(g.params))
        self.entry_structs.append("struct %s {\n%s};\n"
                                  "__device__ void __gtap_entry%d(void* __frame, int __tid, TaskContext* __ctx);\n"
                                  % (ef, fields, k))
        self.entry_defs.append(
            "__device__ void __gtap_entry%d(void* __frame, int __tid, TaskContext* __ctx) {\n"
            "    %s* __f = (%s*)__frame;\n"
            "    switch (__gtap_get_task_state(__tid)) {\n"
            "    case 0: {\n        int __cc = 0;\n"
            "        {\n            %s* __c = (%s*)__gtap_spawn_task(__ctx, __tid, &__cc, %s, 0, nullptr, false);\n"
            "%s            __c->__dst = __gtap_dst(__tid, offsetof(%s, __res));\n        }\n"
            "        if (__gtap_set_state_for_join(__tid, __cc, 1, 0)) return;\n    }\n"
            "    case 1:\n"
            "        %s = __f->__res;\n"
            "        __gtap_finish_task(__tid, __ctx);\n        return;\n"
            "    default:\n        __gtap_finish_task(__tid, __ctx);\n        return;\n    }\n}\n"
            % (k, ef, ef, g.frame, g.frame, g.task, assign, ef, lhs))
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
        # entries, outside the task functions.  An entry task (an entry whose
        # result is assigned) goes right before the kernel that holds the
        # entry, where everything that kernel uses is declared; when the
        # kernel comes before the task functions it goes after the last one.
        out, j = [], 0
        last_task_end = max(f.end for f in self.funcs)
        tail_defs = []
        for pm in PRAGMA.finditer(src):
            if pm.group(1) != "entry":
                continue
            if any(f.start <= pm.start() < f.end for f in self.funcs):
                continue
            n_defs = len(self.entry_defs)
            code, used = self.lower_entry(src[pm.end():], line_of(src, pm.start()))
            head = src[j:pm.start()]
            new_defs = "".join(self.entry_defs[n_defs:])
            g = head.rfind("__global__")
            if new_defs and g >= 0 and j + g >= last_task_end:
                head = head[:g] + new_defs + head[g:]
            else:
                tail_defs.append(new_defs)
            if self.mode == "thread":
                head = self._bound_kernel(head)
            out.append(head)
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
        if self.parent:
            decls += PARENT_HELPERS % size_expr
        # entry tasks, the direct dispatch and the frame size follow the last task function
        tasks = [f.task for f in self.funcs] + ["__gtap_entry%d" % k for k in range(len(self.entry_defs))]
        dispatch = ("__device__ void __gtap_dispatch(unsigned long long __fn, void* __frame, int __tid, "
                    "TaskContext* __ctx) {\n"
                    + "".join("    if (__fn == (unsigned long long)(void*)&%s) { %s(__frame, __tid, __ctx); return; }\n"
                              % (t, t) for t in tasks)
                    + "    ((void (*)(void*, int, TaskContext*))__fn)(__frame, __tid, __ctx);   // a task not lowered here\n"
                    "}\n")
        if self.parent:
            # task functions get the words read with the header; entry tasks read memory
            dispatch = ("__device__ void __gtap_dispatch_words(unsigned long long __fn, void* __frame, int __tid, "
                        "TaskContext* __ctx, int4 __w0, int4 __w1) {\n"
                        + "".join("    if (__fn == (unsigned long long)(void*)&%s) { %s__gtap_run(__frame, __tid, __ctx, "
                                  "__w0, __w1, true); return; }\n" % (f.task, f.name) for f in self.funcs)
                        + "".join("    if (__fn == (unsigned long long)(void*)&__gtap_entry%d) { __gtap_entry%d(__frame, "
                                  "__tid, __ctx); return; }\n" % (k, k) for k in range(len(self.entry_defs)))
                        + "    ((void (*)(void*, int, TaskContext*))__fn)(__frame, __tid, __ctx);   // a task not lowered here\n"
                        "}\n")
        tail = ("".join(tail_defs) + dispatch
                + "const size_t __gtap_auto_task_data_size = %s;\n" % size_expr)
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
        # before any include: the drop-in headers then call the task functions
        # through __gtap_dispatch instead of an indirect call
        if self.parent:
            return "#define GTAP_FRAME_WORDS 1\n#include <cstddef>\n#include <cstring>\n" + "".join(pieces)
        return "#define GTAP_DIRECT_DISPATCH 1\n" + "".join(pieces)


# --results parent: delivering a child's result into its parent's frame, and
# a task's copy of its own frame from the words the worker read with the header
PARENT_HELPERS = """\
constexpr size_t __gtap_frame_max = %s;
// frame bytes the worker loads with the task header: 16, or 32 for frames over 16 bytes
constexpr size_t __gtap_words_bytes = __gtap_frame_max <= 16 ? 16 : 32;
__device__ __forceinline__ unsigned __gtap_dst(int __tid, size_t __offset) {
    return (unsigned)__tid * 32u + (unsigned)(__offset / 4) + 1u;
}
template <typename T>
__device__ __forceinline__ void __gtap_deliver(unsigned __dst, T __v) {
    const unsigned __d = __dst - 1u;
    *reinterpret_cast<T*>(static_cast<char*>(__gtap_get_task_data((int)(__d >> 5))) + 4u * (__d & 31u)) = __v;
}
template <typename F>
__device__ __forceinline__ void __gtap_load_frame(F* __dst, const F* __mem, const int4& __w0, const int4& __w1,
                                                  bool __words) {
    if (!__words) {
        *__dst = *__mem;
        return;
    }
    constexpr size_t __kw = sizeof(F) < __gtap_words_bytes ? sizeof(F) : __gtap_words_bytes;
    const int4 __w[2] = {__w0, __w1};
    memcpy(__dst, __w, __kw);
    if (sizeof(F) > __kw)
        memcpy(reinterpret_cast<char*>(__dst) + __kw, reinterpret_cast<const char*>(__mem) + __kw, sizeof(F) - __kw);
}
"""


def lower_source(src, mode=None, results="retain"):
    """Lowered text of a pragma program; mode 'thread' or 'block' (default:
    from the gtap header it includes).  results 'retain': a parent reads each
    child's result from the child's retained frame after the join (the
    reference's scheme); 'parent' (thread mode): the child writes its result
    into the parent's frame and tasks read their frames from the words the
    worker loads with the task header."""
    if mode is None:
        mode = "block" if re.search(r'#\s*include\s*[<"]gtap_block\.cuh[>"]', src) else "thread"
    if mode not in ("thread", "block"):
        raise LoweringError("mode must be 'thread' or 'block'")
    if results not in ("retain", "parent"):
        raise LoweringError("results must be 'retain' or 'parent'")
    return Lowering(src, mode, results).run()


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("input")
    ap.add_argument("-o", "--output", required=True)
    ap.add_argument("--mode", choices=["thread", "block"], default=None)
    ap.add_argument("--results", choices=["retain", "parent"], default="retain",
                    help="where a child's result goes: its own retained frame, or the parent's frame")
    a = ap.parse_args(argv)
    try:
        with open(a.input) as f:
            out = lower_source(f.read(), a.mode, a.results)
    except LoweringError as e:
        sys.stderr.write("%s: %s\n" % (a.input, e))
        return 1
    with open(a.output, "w") as f:
        f.write(out)
    return 0


if __name__ == "__main__":
    sys.exit(main())
