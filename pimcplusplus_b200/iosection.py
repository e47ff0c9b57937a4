"""PIMC++'s ASCII input format: a reader and writer with IOSectionClass's interface.

Every PIMC++ input — the simulation file, the `.PairAction` files it names,
and any included section file — is a tree of sections holding typed
variables (Common/IO/IOASCII.cc:124-840, Common/IO/IO.cc:101-108):

    double tau = 0.0125;                 // a scalar: double, int, string, bool
    Array<double,1> Box(3) = [14.3, 14.3, 14.3];
    Section (System) {
      Section (Particles) { ... }
    }
    Section (Fits, "other.file");        // a section read from another file

Rules kept from the reference's tokenizer and parser:

* `//` comments run to the end of the line, `/* */` comments may span lines;
  neither is recognised inside a double-quoted string (IOASCII.cc:207-281).
* Tokens are the special characters `(){}[]<>=;,`, quoted strings (no escape
  characters), words (a letter or `_`, then letters, digits and `_`) and
  numbers (a digit, `.` or `-`, then digits, `.`, `e`, `-`, `+`)
  (IOASCII.cc:69-190).  Any other character is an error.
* A scalar value is one token followed by `;`.  A double must be a whole
  `strtod` number, an int a whole base-10 `strtol` number, a bool `true` or
  `false`, a string a quoted token (IOASCII.cc:330-376).
* An array is `Array<type,rank> name(d1,...,dk) = [v, v, ...];` with exactly
  d1*...*dk values, the last index changing fastest (IOASCII.cc:384-500,
  689-745).
* Variables and sections keep their file order; `ReadVar` returns the first
  variable of that name in the current section and `OpenSection(name, n)`
  the n-th section of that name (IO.cc:141-200).

Errors: the reference prints "Error in input file at line number N" and
calls exit(1); here an `InputError` carrying the line number is raised.
`complex` values, which the reference's ASCII reader does not implement
(IOASCII.cc:377-382), are rejected the same way.

Arrays come back as numpy arrays: float64, int64, bool or object (strings).
"""
from __future__ import annotations

import os

import numpy as np

__all__ = ["InputError", "IOTree", "IOSectionClass", "parse_text", "format_tree"]

_SPECIAL = frozenset("(){}[]<>=;,")
_WS = frozenset(" \t\r\n")
_DIGITS = frozenset("0123456789")
_ALPHA = frozenset("abcdefghijklmnopqrstuvwxyzABCDEFGHIJKLMNOPQRSTUVWXYZ_")
_NUM_START = _DIGITS | {".", "-"}
_NUM_CHAR = _DIGITS | {".", "e", "-", "+"}
_TYPES = {"double": np.float64, "int": np.int64, "string": object, "bool": np.bool_}


class InputError(ValueError):
    """A syntax or type error in a PIMC++ input file, with its line number."""

    def __init__(self, line, message, filename=None):
        where = f"{filename}:" if filename else ""
        super().__init__(f"Error in input file {where}line {line}: {message}")
        self.line = line
        self.filename = filename


def _strip_comments(text):
    """Replaces comments with nothing, keeping every newline so line numbers stay."""
    out = []
    i, n = 0, len(text)
    while i < n:
        c = text[i]
        if c == '"':
            j = text.find('"', i + 1)
            j = n - 1 if j < 0 else j
            out.append(text[i:j + 1])
            i = j + 1
        elif text.startswith("//", i):
            j = text.find("\n", i)
            if j < 0:
                break
            i = j  # the newline itself is kept
        elif text.startswith("/*", i):
            j = text.find("*/", i + 2)
            body = text[i:] if j < 0 else text[i:j]
            out.append("\n" * body.count("\n"))
            i = n if j < 0 else j + 2
        else:
            out.append(c)
            i += 1
    return "".join(out)


def _tokenize(text, filename=None):
    """(token, line) pairs; quoted strings keep their quotes."""
    toks = []
    i, n, line = 0, len(text), 1
    while i < n:
        c = text[i]
        if c in _SPECIAL:
            toks.append((c, line))
            i += 1
        elif c == '"':
            j = text.find('"', i + 1)
            if j < 0:
                raise InputError(line, "unterminated string", filename)
            toks.append((text[i:j + 1], line))
            line += text.count("\n", i, j)
            i = j + 1
        elif c in _ALPHA:
            j = i + 1
            while j < n and (text[j] in _ALPHA or text[j] in _DIGITS):
                j += 1
            toks.append((text[i:j], line))
            i = j
        elif c in _WS:
            line += c == "\n"
            i += 1
        elif c in _NUM_START:
            j = i + 1
            while j < n and text[j] in _NUM_CHAR:
                j += 1
            toks.append((text[i:j], line))
            i = j
        elif c == "\0":
            break
        else:
            raise InputError(line, f"unrecognised character {c!r}", filename)
    return toks


def _atom(tok, line, typ, filename):
    if typ is np.float64:
        # strtod on the whole token: Python's float() also takes '_' digit
        # separators, which the tokenizer never puts inside a number token.
        try:
            if "_" in tok:
                raise ValueError
            return float(tok)
        except ValueError:
            raise InputError(line, f"expected a double, found {tok!r}", filename) from None
    if typ is np.int64:
        if not tok or not (tok.isdigit() or (tok[0] == "-" and tok[1:].isdigit())):
            raise InputError(line, f"expected an int, found {tok!r}", filename)
        return int(tok)
    if typ is np.bool_:
        if tok == "true":
            return True
        if tok == "false":
            return False
        raise InputError(line, f"expected true or false, found {tok!r}", filename)
    if len(tok) < 2 or tok[0] != '"' or tok[-1] != '"':
        raise InputError(line, f"expected a quoted string, found {tok!r}", filename)
    return tok[1:-1]


class IOTree:
    """One section: its name, its variables and subsections in file order."""

    def __init__(self, name="Root", parent=None, filename=None):
        self.name = name
        self.parent = parent
        self.filename = filename
        self.vars = []       # [(name, value)]
        self.sections = []   # [IOTree]

    def var(self, name):
        for k, v in self.vars:
            if k == name:
                return v
        return None

    def find(self, name, num=0):
        hits = [s for s in self.sections if s.name == name]
        return hits[num] if 0 <= num < len(hits) else None

    def count(self, name=None):
        return len(self.sections) if name is None else sum(s.name == name for s in self.sections)


class _Parser:
    def __init__(self, toks, filename, base_dir):
        self.toks = toks
        self.i = 0
        self.filename = filename
        self.base_dir = base_dir

    def _line(self):
        if self.i < len(self.toks):
            return self.toks[self.i][1]
        return self.toks[-1][1] if self.toks else 1

    def _next(self, what):
        if self.i >= len(self.toks):
            raise InputError(self._line(), f"unexpected end of file, expected {what}", self.filename)
        t = self.toks[self.i]
        self.i += 1
        return t

    def _expect(self, s):
        tok, line = self._next(repr(s))
        if tok != s:
            raise InputError(line, f"expected {s!r}, found {tok!r}", self.filename)

    def section(self, tree, want_brace):
        while self.i < len(self.toks) and self.toks[self.i][0] != "}":
            tok, line = self.toks[self.i]
            if tok == "Section":
                self.i += 1
                self._expect("(")
                name, _ = self._next("a section name")
                tok2, line2 = self._next("')' or ','")
                if tok2 == ",":
                    ftok, fline = self._next("a file name")
                    fname = _atom(ftok, fline, object, self.filename)
                    self._expect(")")
                    self._expect(";")
                    sub = _read_tree(self._resolve(fname, fline), name, tree)
                elif tok2 == ")":
                    self._expect("{")
                    sub = IOTree(name, tree, self.filename)
                    self.section(sub, True)
                else:
                    raise InputError(line2, f"expected ')' not found, found {tok2!r}", self.filename)
                tree.sections.append(sub)
            else:
                tree.vars.append(self.variable())
        if self.i >= len(self.toks):
            if want_brace:
                raise InputError(self._line(), "unexpected end of file before '}'", self.filename)
        else:
            self.i += 1  # the closing brace (or a stray one at the top level)

    def _resolve(self, fname, line):
        # Relative to the working directory as the reference opens it; failing
        # that, relative to the including file's directory.
        for cand in (fname, os.path.join(self.base_dir, fname)):
            if os.path.exists(cand):
                return cand
        raise InputError(line, f"cannot open included file {fname!r}", self.filename)

    def variable(self):
        tok, line = self._next("a type")
        if tok == "Array":
            return self.array()
        if tok == "complex":
            raise InputError(line, "complex values are not supported by the ASCII format", self.filename)
        typ = _TYPES.get(tok)
        if typ is None:
            raise InputError(line, f"invalid type {tok!r}", self.filename)
        name, _ = self._next("a variable name")
        self._expect("=")
        val, vline = self._next("a value")
        self._expect(";")
        return name, _atom(val, vline, typ, self.filename)

    def array(self):
        self._expect("<")
        tname, tline = self._next("an element type")
        if tname == "complex":
            raise InputError(tline, "complex values are not supported by the ASCII format", self.filename)
        typ = _TYPES.get(tname)
        if typ is None:
            raise InputError(tline, f"array does not have an atomic type: {tname!r}", self.filename)
        self._expect(",")
        rtok, rline = self._next("the rank")
        rank = _atom(rtok, rline, np.int64, self.filename)
        if not 1 <= rank <= 4:
            raise InputError(rline, f"array rank {rank} is outside 1..4", self.filename)
        self._expect(">")
        name, _ = self._next("an array name")
        self._expect("(")
        dims = []
        for d in range(rank):
            dtok, dline = self._next("a dimension")
            dims.append(_atom(dtok, dline, np.int64, self.filename))
            if dims[-1] < 0:
                raise InputError(dline, "negative array dimension", self.filename)
            self._expect(")" if d == rank - 1 else ",")
        self._expect("=")
        self._expect("[")
        total = int(np.prod(dims)) if dims else 0
        vals = []
        for k in range(total):
            vtok, vline = self._next("an array value")
            vals.append(_atom(vtok, vline, typ, self.filename))
            if k != total - 1:
                self._expect(",")
        self._expect("]")
        self._expect(";")
        arr = np.array(vals, dtype=typ).reshape(dims) if total else np.zeros(dims, dtype=typ)
        return name, arr


def parse_text(text, name="Root", parent=None, filename=None, base_dir="."):
    """Parses the text of one file into an IOTree."""
    toks = _tokenize(_strip_comments(text), filename)
    tree = IOTree(name, parent, filename)
    _Parser(toks, filename, base_dir).section(tree, False)
    return tree


def _read_tree(path, name="Root", parent=None):
    with open(path, "r", encoding="latin-1") as f:
        text = f.read()
    return parse_text(text, name, parent, path, os.path.dirname(os.path.abspath(path)))


def _fmt_atom(v):
    if isinstance(v, (bool, np.bool_)):
        return "true" if v else "false"
    if isinstance(v, (int, np.integer)):
        return str(int(v))
    if isinstance(v, (float, np.floating)):
        return repr(float(v))
    return f'"{v}"'


def _type_name(v):
    if isinstance(v, (bool, np.bool_)):
        return "bool"
    if isinstance(v, (int, np.integer)):
        return "int"
    if isinstance(v, (float, np.floating)):
        return "double"
    if isinstance(v, str):
        return "string"
    raise TypeError(f"cannot write a value of type {type(v).__name__}")


def format_tree(tree, indent=0):
    """The ASCII text of a tree, in the syntax the reader takes."""
    pad = "  " * indent
    lines = []
    for name, v in tree.vars:
        if isinstance(v, np.ndarray):
            if v.dtype == object:
                tname = "string"
            elif v.dtype == np.bool_:
                tname = "bool"
            elif np.issubdtype(v.dtype, np.integer):
                tname = "int"
            else:
                tname = "double"
            dims = ",".join(str(d) for d in v.shape)
            body = ", ".join(_fmt_atom(x) for x in v.reshape(-1).tolist())
            lines.append(f"{pad}Array<{tname},{v.ndim}> {name}({dims}) = [{body}];")
        else:
            lines.append(f"{pad}{_type_name(v)} {name} = {_fmt_atom(v)};")
    for s in tree.sections:
        lines.append(f"{pad}Section ({s.name})")
        lines.append(f"{pad}{{")
        inner = format_tree(s, indent + 1)
        if inner:
            lines.append(inner)
        lines.append(f"{pad}}}")
    return "\n".join(lines)


class IOSectionClass:
    """IOSectionClass (Common/IO/IO.h, IO.cc) over the ASCII format.

    The reading methods keep the reference's names and meaning; ReadVar
    returns the value, or None where the reference's ReadVar returns false.
    The writing methods build a tree that WriteFile stores as ASCII.
    """

    def __init__(self):
        self.current = None

    # ---- reading ----
    def OpenFile(self, filename):
        try:
            self.current = _read_tree(filename)
        except FileNotFoundError:
            return False
        return True

    def OpenText(self, text, base_dir="."):
        self.current = parse_text(text, base_dir=base_dir)
        return True

    def CloseFile(self):
        self.current = None

    def OpenSection(self, name, num=0):
        """Opens the num-th section called `name`; an int `name` opens the
        name-th section of any name (IOSectionClass::OpenSection(int))."""
        if isinstance(name, int):
            sub = self.current.sections[name] if 0 <= name < len(self.current.sections) else None
        else:
            sub = self.current.find(name, num)
        if sub is None:
            return False
        self.current = sub
        return True

    def CloseSection(self):
        if self.current.parent is None:
            raise RuntimeError("CloseSection at the root section")
        self.current = self.current.parent

    def CountSections(self, name=None):
        return self.current.count(name)

    def CountVars(self):
        return len(self.current.vars)

    def GetName(self):
        return self.current.name

    def ReadVar(self, name, default=None):
        v = self.current.var(name)
        return default if v is None else v

    def Require(self, name):
        """ReadVar under the reference's assert(): missing variables are errors."""
        v = self.current.var(name)
        if v is None:
            where = self.current.filename or "input"
            raise InputError(0, f"required variable {name!r} missing in section {self.current.name!r}", where)
        return v

    # ---- writing ----
    def NewFile(self, filename=None):
        self.current = IOTree("Root", None, filename)
        return True

    def NewSection(self, name):
        sub = IOTree(name, self.current, self.current.filename)
        self.current.sections.append(sub)
        self.current = sub

    def WriteVar(self, name, value):
        if isinstance(value, (list, tuple)):
            value = np.array(value)
        self.current.vars.append((name, value))

    def WriteFile(self, filename):
        root = self.current
        while root.parent is not None:
            root = root.parent
        with open(filename, "w") as f:
            f.write(format_tree(root) + "\n")
