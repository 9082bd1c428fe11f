"""File front end: PDB / mmCIF / XYZR input, atomic radii, VMD-like selections, and
compute_tessellation_from_file (src/input/*.rs, src/python.rs:266-324).

Host-side parsing in front of the GPU tessellation: a structure file becomes an (N, 4)
ball array (radius by residue and atom name) and, for selections, the per-atom records
the selection language matches.  The rules follow the reference:

* format by extension (.pdb .ent .pdb1 / .cif .mmcif / .xyzr), else by the first line
  (mod.rs:80-118);
* PDB: fixed columns, ATOM/HETATM; first model only unless ``as_assembly`` (then the
  model number is appended to the chain id of models > 1); stops at END (pdb.rs);
* mmCIF: the ``_atom_site`` loop, auth fields with label fallbacks, first model only
  unless ``as_assembly`` (mmcif.rs);
* both drop alternate locations other than A / 1 / ".", hydrogens (unless asked for)
  and waters; atom names with leading digits are rotated ("1HB" -> "HB1");
* radii: an exact (residue, atom) rule, then the longest matching "prefix*" rule, first
  for the residue and then for "*", then a (residue, "*") / ("*", "*") rule, else 1.80
  (radii.rs:58-85); the default rules are radii_default.txt;
* selections: ``and or not ( )``, ``chain resname resid name`` with glob patterns
  (* ? [a-z]) and resid ranges (``1 to 9``, ``1:9``), and residue classes
  (selection.rs); with group selections, an atom's group is the first selection that
  matches it, unmatched atoms each get a group of their own (selection.rs:773-813).
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field

import numpy as np

DEFAULT_RADIUS = 1.8
_HERE = os.path.dirname(os.path.abspath(__file__))


# ---- records ------------------------------------------------------------------------
@dataclass
class AtomRecord:
    record_name: str
    serial: int
    name: str
    alt_loc: str
    res_name: str
    chain_id: str
    res_seq: int
    i_code: str
    x: float
    y: float
    z: float
    element: str
    b_factor: float = 0.0


@dataclass
class ParseOptions:
    exclude_heteroatoms: bool = False
    include_hydrogens: bool = False
    as_assembly: bool = False


@dataclass
class ParsedStructure:
    balls: np.ndarray  # (N, 4) x y z r
    records: list = field(default_factory=list)  # empty for XYZR


def _undef(s: str) -> str:
    return "" if s in (".", "?") else s


def _rotate_name(name: str) -> str:
    """Leading digits move to the end ("1HB" -> "HB1"); all-digit names stay."""
    for k, ch in enumerate(name):
        if not ch.isdigit():
            return name if k == 0 else name[k:] + name[:k]
    return name


def _acceptable(r: AtomRecord, opt: ParseOptions) -> bool:
    if r.record_name == "HETATM" and opt.exclude_heteroatoms:
        return False
    if r.alt_loc not in ("", "A", "1", "."):
        return False
    if not opt.include_hydrogens and (r.name.startswith("H") or r.element in ("H", "D")):
        return False
    return r.res_name != "HOH"


def _int(s: str):
    try:
        return int(s)
    except ValueError:
        return None


def _float(s: str):
    try:
        return float(s)
    except ValueError:
        return None


# ---- PDB ----------------------------------------------------------------------------
def _col(line: str, start: int, end: int) -> str:
    """1-based inclusive columns, trimmed (pdb.rs:15-27)."""
    return line[start - 1:end].strip() if start - 1 < len(line) else ""


def _pdb_atom(line: str):
    rec = _col(line, 1, 6)
    if rec not in ("ATOM", "HETATM"):
        return None
    xs, ys, zs = _col(line, 31, 38), _col(line, 39, 46), _col(line, 47, 54)
    x, y, z = _float(xs) if xs else None, _float(ys) if ys else None, _float(zs) if zs else None
    serial = _int(_col(line, 7, 11))
    res_seq = _int(_col(line, 23, 26))
    name = _col(line, 13, 16)
    if None in (x, y, z, serial, res_seq) or not name:
        return None
    b = _col(line, 61, 66)
    bf = _float(b) if b else None
    return AtomRecord(rec, serial, _rotate_name(name), _undef(_col(line, 17, 17)), _undef(_col(line, 18, 20)),
                      _undef(_col(line, 22, 22)), res_seq, _undef(_col(line, 27, 27)), x, y, z,
                      _undef(_col(line, 77, 78)), 0.0 if bf is None else bf)


def parse_pdb(lines, options: ParseOptions | None = None) -> list:
    opt = options or ParseOptions()
    out, model = [], 1
    for line in lines:
        line = line.rstrip("\r\n")
        rec = _col(line, 1, 6)
        if rec in ("ATOM", "HETATM"):
            r = _pdb_atom(line)
            if r is not None and _acceptable(r, opt):
                if opt.as_assembly and model > 1:
                    r.chain_id = f"{r.chain_id}{model}"
                r.alt_loc = ""
                out.append(r)
        elif rec == "ENDMDL":
            model += 1
            if not opt.as_assembly:
                break
        elif rec == "END":
            break
    return out


# ---- mmCIF --------------------------------------------------------------------------
def _cif_tokens(lines):
    """Whitespace-separated tokens; quoted tokens keep their spaces; # starts a comment."""
    for line in lines:
        i, n = 0, len(line)
        while i < n:
            ch = line[i]
            if ch.isspace():
                i += 1
                continue
            if ch == "#":
                break
            if ch in "'\"":
                j = line.find(ch, i + 1)
                j = n if j < 0 else j
                yield line[i + 1:j]
                i = j + 1
                continue
            j = i
            while j < n and not line[j].isspace():
                j += 1
            yield line[i:j]
            i = j


_CIF_FIELDS = ("pdbx_PDB_model_num", "group_PDB", "id", "auth_atom_id", "label_atom_id", "label_alt_id",
               "auth_comp_id", "label_comp_id", "auth_asym_id", "label_asym_id", "auth_seq_id", "label_seq_id",
               "pdbx_PDB_ins_code", "Cartn_x", "Cartn_y", "Cartn_z", "type_symbol", "B_iso_or_equiv")


def _cif_row(row, fmap):
    def get(primary, fallback=None):
        k = fmap.get(primary)
        if k is not None and k < len(row):
            return row[k]
        k = fmap.get(fallback) if fallback else None
        if k is not None and k < len(row):
            return row[k]
        return ""

    x, y, z = _float(get("Cartn_x")), _float(get("Cartn_y")), _float(get("Cartn_z"))
    serial = _int(get("id"))
    res_seq = _int(get("auth_seq_id", "label_seq_id"))
    name = get("auth_atom_id", "label_atom_id")
    rec = get("group_PDB")
    if None in (x, y, z, serial, res_seq) or not name or not rec:
        return None
    bf = _float(get("B_iso_or_equiv"))
    return AtomRecord(rec, serial, _rotate_name(name), _undef(get("label_alt_id")),
                      _undef(get("auth_comp_id", "label_comp_id")), _undef(get("auth_asym_id", "label_asym_id")),
                      res_seq, _undef(get("pdbx_PDB_ins_code")), x, y, z, _undef(get("type_symbol")),
                      0.0 if bf is None else bf)


def parse_mmcif(lines, options: ParseOptions | None = None) -> list:
    opt = options or ParseOptions()
    toks = _cif_tokens(lines)
    out = []
    for tok in toks:
        if tok != "loop_":
            continue
        header, fmap = [], {}
        first = None
        for t in toks:
            if not t.startswith("_atom_site."):
                first = t
                break
            name = t[len("_atom_site."):]
            if name in _CIF_FIELDS:
                fmap[name] = len(header)
            header.append(t)
        if not header or first is None:
            continue
        ncol, first_model = len(header), None
        row = [first]
        while True:
            while len(row) < ncol:
                t = next(toks, None)
                if t is None:
                    return out
                row.append(t)
            if row[0].startswith("_") or row[0].startswith("data_") or row[0] == "loop_":
                break
            k = fmap.get("pdbx_PDB_model_num")
            model = row[k] if k is not None and k < len(row) else ""
            if first_model is None:
                first_model = model
            if opt.as_assembly or model == first_model:
                r = _cif_row(row, fmap)
                if r is not None and _acceptable(r, opt):
                    if opt.as_assembly and model not in ("1", ""):
                        r.chain_id = f"{r.chain_id}{model}"
                    r.alt_loc = ""
                    out.append(r)
            t = next(toks, None)
            if t is None:
                return out
            row = [t]
        # a new loop_ / data block / item starts at row[0]: the outer scan resumes after it
    return out


# ---- XYZR ---------------------------------------------------------------------------
def parse_xyzr(lines) -> np.ndarray:
    """x y z r as the last four numbers of each line (other lines skipped)."""
    rows = []
    for line in lines:
        parts = line.split()
        if len(parts) < 4:
            continue
        vals = [_float(p) for p in parts[-4:]]
        if None in vals:
            continue
        rows.append(vals)
    return np.array(rows, dtype=np.float64).reshape(-1, 4)


# ---- radii --------------------------------------------------------------------------
class RadiiLookup:
    """Radius by (residue name, atom name) rules (radii.rs)."""

    def __init__(self, rules: dict | None = None):
        self.rules = dict(rules or {})

    @classmethod
    def default(cls) -> "RadiiLookup":
        r = cls()
        with open(os.path.join(_HERE, "radii_default.txt")) as f:
            r.load_text(f.read())
        return r

    def load_text(self, text: str) -> None:
        """Rules "residue atom radius" per line ('#' comments); later rules replace
        earlier ones with the same key."""
        for line in text.splitlines():
            line = line.strip()
            if not line or line.startswith("#"):
                continue
            parts = line.split()
            if len(parts) < 3:
                raise ValueError(f"Invalid radii rule: {line}")
            r = _float(parts[2])
            if r is None:
                raise ValueError(f"Invalid radius value: {parts[2]}")
            if r < 0.0:
                raise ValueError(f"Negative radius: {r}")
            self.rules[(parts[0], parts[1])] = r

    def radius(self, res_name: str, atom_name: str) -> float:
        if not atom_name or atom_name == "*":
            return DEFAULT_RADIUS
        get = self.rules.get
        for res in (res_name, "*"):
            v = get((res, atom_name))
            if v is not None:
                return v
            for k in range(len(atom_name), 0, -1):
                v = get((res, atom_name[:k] + "*"))
                if v is not None:
                    return v
        for res in (res_name, "*"):
            v = get((res, "*"))
            if v is not None:
                return v
        return DEFAULT_RADIUS


# ---- format detection and parse_file ------------------------------------------------
_EXT = {"pdb": "pdb", "ent": "pdb", "pdb1": "pdb", "cif": "mmcif", "mmcif": "mmcif", "xyzr": "xyzr"}


def detect_format(path: str, first_line: str | None) -> str | None:
    ext = os.path.splitext(path)[1][1:].lower()
    if ext in _EXT:
        return _EXT[ext]
    if first_line is None:
        return None
    t = first_line.strip()
    if t.startswith("data_") or t.startswith("_") or t.startswith("loop_"):
        return "mmcif"
    if t.startswith(("ATOM", "HETATM", "HEADER", "REMARK")):
        return "pdb"
    parts = t.split()
    if len(parts) >= 4 and all(_float(p) is not None for p in parts[-4:]):
        return "xyzr"
    return None


def _open_text(path: str):
    if path.endswith(".gz"):
        import gzip
        return gzip.open(path, "rt")
    return open(path)


def parse_file(path: str, options: ParseOptions | None = None, radii: RadiiLookup | None = None) -> ParsedStructure:
    """Balls (and atom records for PDB / mmCIF) of a structure file.  A ".gz" suffix is
    read through gzip; the format comes from the name without it.  Raises OSError."""
    radii = radii or RadiiLookup.default()
    with _open_text(path) as f:
        lines = f.read().splitlines()
    name = path[:-3] if path.endswith(".gz") else path
    fmt = detect_format(name, next((l for l in lines[:1]), None))
    if fmt is None:
        raise OSError("Unable to detect input format")
    if fmt == "xyzr":
        return ParsedStructure(parse_xyzr(lines), [])
    recs = parse_pdb(lines, options) if fmt == "pdb" else parse_mmcif(lines, options)
    balls = np.array([(r.x, r.y, r.z, radii.radius(r.res_name, r.name)) for r in recs],
                     dtype=np.float64).reshape(-1, 4)
    return ParsedStructure(balls, recs)


# ---- groupings ----------------------------------------------------------------------
def build_chain_grouping(records) -> np.ndarray:
    ids: dict = {}
    return np.array([ids.setdefault(r.chain_id, len(ids)) for r in records], dtype=np.int32)


def build_residue_grouping(records) -> np.ndarray:
    ids: dict = {}
    return np.array([ids.setdefault((r.chain_id, r.res_seq, r.i_code), len(ids)) for r in records], dtype=np.int32)


# ---- selections ---------------------------------------------------------------------
class SelectionError(ValueError):
    def __init__(self, message: str, position: int):
        super().__init__(f"{message} at position {position}")
        self.message, self.position = message, position


def glob_match(pattern: str, text: str) -> bool:
    """* (any run), ? (any one), [abc] / [a-z] classes; backtracking to the last star."""
    p = t = 0
    star_p = star_t = -1
    while t < len(text):
        if p < len(pattern):
            c = pattern[p]
            if c == "?":
                p += 1
                t += 1
                continue
            if c == "*":
                star_p, star_t = p, t
                p += 1
                continue
            if c == "[":
                cls = _char_class(pattern, p, text[t])
                if cls is not None and cls[0]:
                    p = cls[1] + 1
                    t += 1
                    continue
            elif c == text[t]:
                p += 1
                t += 1
                continue
        if star_p < 0:
            return False
        p = star_p + 1
        star_t += 1
        t = star_t
    while p < len(pattern) and pattern[p] == "*":
        p += 1
    return p == len(pattern)


def _char_class(pattern: str, start: int, ch: str):
    i, hit = start + 1, False
    while i < len(pattern) and pattern[i] != "]":
        if i + 2 < len(pattern) and pattern[i + 1] == "-" and pattern[i + 2] != "]":
            hit = hit or pattern[i] <= ch <= pattern[i + 2]
            i += 3
        else:
            hit = hit or pattern[i] == ch
            i += 1
    return (hit, i) if i < len(pattern) else None


_PROTEIN = {"ALA", "ARG", "ASN", "ASP", "CYS", "GLN", "GLU", "GLY", "HIS", "ILE", "LEU", "LYS", "MET", "PHE",
            "PRO", "SER", "THR", "TRP", "TYR", "VAL", "HIE", "HID", "HIP", "CYX", "ASH", "GLH", "LYN"}
_NUCLEIC = {"DA", "DT", "DG", "DC", "DU", "A", "U", "G", "C", "RA", "RU", "RG", "RC"}
_BACKBONE = {"C", "CA", "N", "O"}
_HYDROPHOBIC = {"ALA", "VAL", "ILE", "LEU", "MET", "PHE", "TRP", "PRO", "GLY"}
_AROMATIC = {"PHE", "TYR", "TRP", "HIS", "HIE", "HID", "HIP"}
_ACIDIC = {"ASP", "GLU", "ASH", "GLH"}
_BASIC = {"ARG", "LYS", "HIS", "HIE", "HID", "HIP", "LYN"}
_POLAR = {"SER", "THR", "ASN", "GLN", "CYS", "CYX", "TYR"}
_CLASSES = {
    "protein": lambda r: r.res_name in _PROTEIN,
    "backbone": lambda r: r.res_name in _PROTEIN and r.name in _BACKBONE,
    "sidechain": lambda r: r.res_name in _PROTEIN and r.name not in _BACKBONE,
    "nucleic": lambda r: r.res_name in _NUCLEIC,
    "hetatm": lambda r: r.record_name == "HETATM",
    "hydrophobic": lambda r: r.res_name in _HYDROPHOBIC,
    "aromatic": lambda r: r.res_name in _AROMATIC,
    "acidic": lambda r: r.res_name in _ACIDIC,
    "basic": lambda r: r.res_name in _BASIC,
    "polar": lambda r: r.res_name in _POLAR,
    "charged": lambda r: r.res_name in _ACIDIC or r.res_name in _BASIC,
    "all": lambda r: True,
    "none": lambda r: False,
}
_KEYWORDS = {"chain": "chain", "segid": "chain", "resname": "resname", "resn": "resname", "resid": "resid",
             "resi": "resid", "resseq": "resid", "resnum": "resid", "name": "name", "atomname": "name",
             "nucleicacid": "nucleic", "hetero": "hetatm", "everything": "all", "nothing": "none",
             "and": "and", "&&": "and", "or": "or", "||": "or", "not": "not", "!": "not", "to": "to"}
_KEYWORDS.update({k: k for k in _CLASSES})


def _tokenize(text: str):
    toks, i, n = [], 0, len(text)
    ident_start = lambda c: c.isascii() and (c.isalnum() or c in "_*?['")  # noqa: E731
    while i < n:
        c = text[i]
        if c.isspace():
            i += 1
        elif c in "():":
            toks.append(({"(": "(", ")": ")", ":": ":"}[c], None, i))
            i += 1
        elif c in "\"'":
            j = text.find(c, i + 1)
            j = n if j < 0 else j
            toks.append(("id", text[i + 1:j], i + 1))
            i = j + 1
        elif c.isdigit() or (c == "-" and i + 1 < n and text[i + 1].isdigit()):
            j = i + 1
            while j < n and text[j].isdigit():
                j += 1
            toks.append(("num", int(text[i:j]), i))
            i = j
        elif ident_start(c):
            j, in_br = i, False
            while j < n:
                ch = text[j]
                if ch == "[":
                    in_br = True
                elif ch == "]":
                    in_br = False
                if in_br or (ch.isascii() and (ch.isalnum() or ch in "_*?[]-'")):
                    j += 1
                else:
                    break
            word = text[i:j]
            kw = _KEYWORDS.get(word.lower())
            toks.append((kw, None, i) if kw else ("id", word, i))
            i = j
        else:
            raise SelectionError(f"Unexpected character: {c}", i)
    return toks


class Selection:
    """A parsed selection; ``matches(record)``."""

    def __init__(self, text: str):
        self.text = text
        self._t = _tokenize(text)
        self._k = 0
        if not self._t:
            raise SelectionError("Empty selection", 0)
        self._fn = self._or()
        if self._k < len(self._t):
            raise SelectionError("Unexpected token after expression", self._pos())

    def matches(self, record) -> bool:
        return self._fn(record)

    def _peek(self):
        return self._t[self._k][0] if self._k < len(self._t) else None

    def _pos(self):
        return self._t[self._k][2] if self._k < len(self._t) else 0

    def _or(self):
        left = self._and()
        while self._peek() == "or":
            self._k += 1
            right = self._and()
            left = (lambda a, b: lambda r: a(r) or b(r))(left, right)
        return left

    def _and(self):
        left = self._not()
        while self._peek() == "and":
            self._k += 1
            right = self._not()
            left = (lambda a, b: lambda r: a(r) and b(r))(left, right)
        return left

    def _not(self):
        if self._peek() == "not":
            self._k += 1
            inner = self._not()
            return lambda r: not inner(r)
        return self._primary()

    def _primary(self):
        kind, pos = self._peek(), self._pos()
        if kind == "(":
            self._k += 1
            inner = self._or()
            if self._peek() != ")":
                raise SelectionError("Missing closing parenthesis", self._pos())
            self._k += 1
            return inner
        if kind in ("chain", "resname", "name"):
            self._k += 1
            pats = []
            while self._peek() == "id":
                pats.append(self._t[self._k][1])
                self._k += 1
            if not pats:
                raise SelectionError(f"{kind} requires at least one argument", pos)
            attr = {"chain": "chain_id", "resname": "res_name", "name": "name"}[kind]
            return lambda r: any(glob_match(p, getattr(r, attr)) for p in pats)
        if kind == "resid":
            self._k += 1
            ranges = self._ranges()
            if not ranges:
                raise SelectionError("resid requires at least one argument", pos)
            return lambda r: any(lo <= r.res_seq <= hi for lo, hi in ranges)
        if kind in _CLASSES:
            self._k += 1
            return _CLASSES[kind]
        if kind in ("and", "or"):
            raise SelectionError("Unexpected boolean operator", pos)
        if kind == "id":
            raise SelectionError(f"Unknown keyword: {self._t[self._k][1]}", pos)
        raise SelectionError("Expected selection expression", pos)

    def _ranges(self):
        out = []
        while self._k < len(self._t):
            kind, val, _ = self._t[self._k]
            if kind == "num":
                self._k += 1
                if self._peek() in ("to", ":"):
                    self._k += 1
                    if self._peek() != "num":
                        sep = "'to'" if self._t[self._k - 1][0] == "to" else "':'"
                        raise SelectionError(f"Expected number after {sep}", self._pos())
                    out.append((val, self._t[self._k][1]))
                    self._k += 1
                else:
                    out.append((val, val))
            elif kind == "id":
                parts = val.split(":")
                if len(parts) == 2 and _int(parts[0]) is not None and _int(parts[1]) is not None:
                    out.append((int(parts[0]), int(parts[1])))
                elif _int(val) is not None:
                    out.append((int(val), int(val)))
                else:
                    break
                self._k += 1
            else:
                break
        return out


def parse_selections(texts) -> list:
    if len(texts) < 2:
        raise SelectionError("At least two selections required", 0)
    out = []
    for idx, t in enumerate(texts):
        try:
            out.append(Selection(t.strip()))
        except SelectionError as e:
            raise SelectionError(e.message, idx) from None
    return out


def build_custom_grouping(records, selections) -> np.ndarray:
    """Group of the first selection an atom matches; unmatched atoms get unique groups
    numbered after the selections, in atom order."""
    groups = np.full(len(records), -1, dtype=np.int32)
    for i, r in enumerate(records):
        for g, s in enumerate(selections):
            if s.matches(r):
                groups[i] = g
                break
    unmatched = np.nonzero(groups < 0)[0]
    groups[unmatched] = len(selections) + np.arange(len(unmatched), dtype=np.int32)
    return groups


# ---- compute_tessellation_from_file ---------------------------------------------------
def compute_tessellation_from_file(path, probe, periodic_box=None, with_cell_vertices=False, group_selections=None,
                                   precision="fp32", radii: RadiiLookup | None = None,
                                   options: ParseOptions | None = None) -> dict:
    """compute_tessellation_from_file (mod.rs:544-573, python.rs:266-324): parse, group by
    selections (at least two), tessellate on the GPU; the reference's result dict.  Every
    failure of the file part raises OSError (IOError), as the reference's binding does."""
    from . import compute_tessellation

    if group_selections is not None and len(group_selections) < 2:
        raise OSError("at least two selections required for grouping")
    try:
        parsed = parse_file(str(path), options, radii)
    except OSError as e:
        raise OSError(f"I/O error: {e}") from e
    groups = None
    if group_selections is not None:
        if not parsed.records:
            raise OSError("selections require PDB or mmCIF input (not XYZR)")
        try:
            sels = parse_selections(list(group_selections))
        except SelectionError as e:
            raise OSError(f"selection error: {e}") from e
        groups = build_custom_grouping(parsed.records, sels)
    return compute_tessellation(parsed.balls, probe, periodic_box, groups, with_cell_vertices, precision)
