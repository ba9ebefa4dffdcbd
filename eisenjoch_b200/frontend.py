"""Netlist ingestion: Yosys JSON -> design -> the placer's flat CSR form.

Mirrors the reference's frontend (crates/nextpnr/src/frontend/mod.rs) and
the flattening its placer performs when it walks a Context
(collect_movable_cells, placer/common.rs:155-174; pins of a net = driver,
then users, netlist/net.rs:14-67; add_wa_wirelength_gradient,
placer/common.rs:205-291), so a design synthesised by Yosys can be placed by
this library.

Behaviour kept from the reference, and why it matters here:
  * serde_json is used without `preserve_order`, so every JSON object is a
    sorted map: modules, cells, ports, connections, netnames are visited in
    sorted key order.  Cell creation order is the solver order of the
    placer, so this module sorts keys the same way.
  * One net per signal bit, created in first-appearance order (cells, then
    top-level ports); then the constant nets $PACKER_GND_NET and
    $PACKER_VCC_NET and their driver cells $PACKER_GND / $PACKER_VCC (type
    GND / VCC, output Y); then the cells; then one pseudo-cell per top-level
    port bit ($io$<name>, type $nextpnr_IBUF / $nextpnr_OBUF /
    $nextpnr_IOBUF, internal port O / I / IO); then the netnames.
  * Multi-bit ports and netnames get indexed names `name[i]`; constant bits
    "0" / "1" connect to the GND / VCC nets, "x" / "z" stay unconnected.
  * An output port drives its net (a later driver replaces an earlier one),
    input and inout ports become users, in connection order.
  * Port directions come from `port_directions`, else from the cell type and
    port name (LUT4: F drives; CARRY4: CO* and O* drive; GND / VCC / *_DRV
    drive; IOB is inout; otherwise Q, O, F and Y drive).
  * The top module is the first (in sorted order) whose `top` attribute is a
    non-zero integer, else the first module.
  * Netnames with hide_name != 0 are not applied.
Errors raise ValueError with the reference's messages.

Flattening to the placer's input (a chip model with one logic BEL per site
and IO BELs on the periphery, as the rest of this library uses): the logic
cells are movable, in creation order; the IO pseudo-cells are fixed pads at
the given locations (by default evenly spaced along the chip's perimeter);
the constant nets are left out, their drivers being global resources rather
than placed cells.
"""

import json
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

import numpy as np

IN, OUT, INOUT = "in", "out", "inout"
IO_TYPES = {"$nextpnr_IBUF", "$nextpnr_OBUF", "$nextpnr_IOBUF"}
GND_NET, VCC_NET = "$PACKER_GND_NET", "$PACKER_VCC_NET"


@dataclass
class Port:
    direction: str
    net: Optional[int] = None
    user_index: Optional[int] = None


@dataclass
class Cell:
    name: str
    type: str
    ports: Dict[str, Port] = field(default_factory=dict)
    params: Dict[str, object] = field(default_factory=dict)
    attrs: Dict[str, object] = field(default_factory=dict)


@dataclass
class Net:
    name: str
    driver: Optional[Tuple[int, str]] = None       # (cell index, port)
    users: List[Tuple[int, str]] = field(default_factory=list)
    attrs: Dict[str, object] = field(default_factory=dict)


@dataclass
class Design:
    top_module: str = ""
    cells: List[Cell] = field(default_factory=list)
    nets: List[Net] = field(default_factory=list)

    def cell(self, name):
        for c in self.cells:
            if c.name == name:
                return c
        return None

    def net(self, name):
        for n in self.nets:
            if n.name == name:
                return n
        return None


# --- helpers (frontend/mod.rs: parse_bit_value, parse_port_direction, ...) --
def parse_bit_value(v):
    """An int is a signal index; "0" / "1" constants; "x" / "z" undefined."""
    if isinstance(v, bool):
        raise ValueError("Invalid bit value in connections array: %r" % (v,))
    if isinstance(v, int):
        return ("signal", v)
    if isinstance(v, str):
        if v == "0":
            return ("zero", None)
        if v == "1":
            return ("one", None)
        if v in ("x", "z"):
            return ("undef", None)
        raise ValueError("Unknown constant bit value: %r" % v)
    raise ValueError("Invalid bit value in connections array: %r" % (v,))


def parse_port_direction(s):
    try:
        return {"input": IN, "output": OUT, "inout": INOUT}[s]
    except KeyError:
        raise ValueError("Unknown port direction: %r" % s) from None


def infer_port_direction(cell_type, port):
    if cell_type == "LUT4":
        return OUT if port == "F" else IN
    if cell_type == "CARRY4":
        return OUT if port.startswith("CO") or port.startswith("O") else IN
    if cell_type in ("GND", "VCC", "GND_DRV", "VCC_DRV"):
        return OUT
    if cell_type == "IOB":
        return INOUT
    return OUT if port in ("Q", "O", "F", "Y") else IN


def parse_property(v):
    """Ints stay ints; strings of only '0'/'1' are bit vectors (kept as
    ('bits', s)); other strings stay strings."""
    if isinstance(v, bool) or not isinstance(v, (int, str)):
        raise ValueError("Unsupported property value type: %r" % (v,))
    if isinstance(v, int):
        return v
    if v and all(ch in "01" for ch in v):
        return ("bits", v)
    return v


def property_as_int(p):
    if isinstance(p, int):
        return p
    if isinstance(p, tuple) and p[0] == "bits":
        return int(p[1], 2)
    if isinstance(p, str):
        try:
            return int(p)
        except ValueError:
            return None
    return None


def port_bit_name(base, i, total):
    return base if total == 1 else "%s[%d]" % (base, i)


def _sorted_items(obj):
    # serde_json's default map is a BTreeMap: keys in byte order
    return sorted(obj.items(), key=lambda kv: kv[0].encode("utf-8"))


# --- parsing ------------------------------------------------------------------
def parse_yosys_json(text):
    """parse_json (frontend/mod.rs): the design of the top module."""
    try:
        doc = json.loads(text)
    except json.JSONDecodeError as e:
        raise ValueError("Failed to parse JSON: %s" % e) from None
    modules = doc.get("modules") if isinstance(doc, dict) else None
    if not isinstance(modules, dict):
        raise ValueError("Missing or invalid 'modules' key in JSON")
    if not modules:
        raise ValueError("No modules found in JSON")
    mods = _sorted_items(modules)
    top_name, top = mods[0]
    for name, m in mods:
        attrs = m.get("attributes") if isinstance(m, dict) else None
        if isinstance(attrs, dict) and "top" in attrs:
            v = property_as_int(parse_property(attrs["top"]))
            if v:
                top_name, top = name, m
                break
    d = Design(top_module=top_name)
    try:
        _parse_module(top, d)
    except ValueError as e:
        raise ValueError("Failed to parse module '%s': %s" % (top_name, e)) from None
    return d


def _connect(d, ci, port, direction, ni):
    c, n = d.cells[ci], d.nets[ni]
    if direction == OUT:
        c.ports[port].net = ni
        c.ports[port].user_index = None
        n.driver = (ci, port)
    else:
        n.users.append((ci, port))
        c.ports[port].net = ni
        c.ports[port].user_index = len(n.users) - 1


def _parse_module(m, d):
    bit_to_net = {}

    def add_signal(idx):
        if idx not in bit_to_net:
            bit_to_net[idx] = len(d.nets)
            d.nets.append(Net("$signal$%d" % idx))

    cells = m.get("cells") if isinstance(m.get("cells"), dict) else {}
    ports = m.get("ports") if isinstance(m.get("ports"), dict) else {}
    for _, cj in _sorted_items(cells):
        conns = cj.get("connections")
        if isinstance(conns, dict):
            for _, bits in _sorted_items(conns):
                if not isinstance(bits, list):
                    raise ValueError("Cell connection bits must be an array")
                for b in bits:
                    kind, idx = parse_bit_value(b)
                    if kind == "signal":
                        add_signal(idx)
    for _, pj in _sorted_items(ports):
        bits = pj.get("bits")
        if isinstance(bits, list):
            for b in bits:
                kind, idx = parse_bit_value(b)
                if kind == "signal":
                    add_signal(idx)
    gnd = len(d.nets)
    d.nets.append(Net(GND_NET))
    vcc = len(d.nets)
    d.nets.append(Net(VCC_NET))
    for cname, ctype, ni in (("$PACKER_GND", "GND", gnd), ("$PACKER_VCC", "VCC", vcc)):
        d.cells.append(Cell(cname, ctype, {"Y": Port(OUT)}))
        _connect(d, len(d.cells) - 1, "Y", OUT, ni)

    def net_of(kind, idx):
        if kind == "signal":
            if idx not in bit_to_net:
                raise ValueError("Signal bit index not found in net map")
            return bit_to_net[idx]
        return {"zero": gnd, "one": vcc}.get(kind)

    for cname, cj in _sorted_items(cells):
        ctype = cj.get("type")
        if not isinstance(ctype, str):
            raise ValueError("Failed to parse cell '%s': Cell missing 'type' field" % cname)
        d.cells.append(Cell(cname, ctype))
        ci = len(d.cells) - 1
        dirs = {}
        pdirs = cj.get("port_directions")
        if isinstance(pdirs, dict):
            for pname, dv in _sorted_items(pdirs):
                if not isinstance(dv, str):
                    raise ValueError("port_direction value must be a string")
                dirs[pname] = parse_port_direction(dv)
        conns = cj.get("connections")
        if isinstance(conns, dict):
            for pname, bits in _sorted_items(conns):
                if not isinstance(bits, list):
                    raise ValueError("Connection bits must be an array")
                direction = dirs.get(pname) or infer_port_direction(ctype, pname)
                for i, b in enumerate(bits):
                    kind, idx = parse_bit_value(b)
                    name = port_bit_name(pname, i, len(bits))
                    d.cells[ci].ports.setdefault(name, Port(direction))
                    ni = net_of(kind, idx)
                    if ni is not None:
                        _connect(d, ci, name, direction, ni)
        for key, target in (("parameters", d.cells[ci].params), ("attributes", d.cells[ci].attrs)):
            obj = cj.get(key)
            if isinstance(obj, dict):
                for k, v in _sorted_items(obj):
                    target[k] = parse_property(v)

    for pname, pj in _sorted_items(ports):
        dv = pj.get("direction")
        if not isinstance(dv, str):
            raise ValueError("Top-level port missing 'direction'")
        direction = parse_port_direction(dv)
        bits = pj.get("bits")
        if not isinstance(bits, list):
            raise ValueError("Top-level port missing 'bits'")
        ctype, iport, idir = {IN: ("$nextpnr_IBUF", "O", OUT), OUT: ("$nextpnr_OBUF", "I", IN),
                              INOUT: ("$nextpnr_IOBUF", "IO", INOUT)}[direction]
        for i, b in enumerate(bits):
            kind, idx = parse_bit_value(b)
            d.cells.append(Cell("$io$" + port_bit_name(pname, i, len(bits)), ctype, {iport: Port(idir)}))
            ni = net_of(kind, idx)
            if ni is not None:
                _connect(d, len(d.cells) - 1, iport, idir, ni)

    netnames = m.get("netnames")
    if isinstance(netnames, dict):
        for nname, nj in _sorted_items(netnames):
            hide = nj.get("hide_name", 0)
            if isinstance(hide, int) and hide != 0:
                continue
            bits = nj.get("bits")
            if not isinstance(bits, list):
                raise ValueError("netnames entry missing 'bits'")
            for i, b in enumerate(bits):
                kind, idx = parse_bit_value(b)
                if kind == "signal" and idx in bit_to_net:
                    d.nets[bit_to_net[idx]].name = port_bit_name(nname, i, len(bits))
            attrs = nj.get("attributes")
            if isinstance(attrs, dict) and bits:
                kind, idx = parse_bit_value(bits[0])
                if kind == "signal" and idx in bit_to_net:
                    for k, v in _sorted_items(attrs):
                        d.nets[bit_to_net[idx]].attrs[k] = parse_property(v)


# --- flattening ---------------------------------------------------------------
def perimeter_sites(count, width, height):
    """`count` sites evenly spaced along the chip's perimeter walk (x along
    the bottom, up the right edge, back along the top, down the left edge),
    the pad placement of this library's benchmark netlists."""
    L = 2 * width + 2 * height - 4 if height >= 2 else width
    out = []
    for f in range(count):
        p = f * L // max(count, 1)
        if p < width:
            xy = (p, 0)
        elif p < width + height - 1:
            xy = (width - 1, p - width + 1)
        elif p < 2 * width + height - 2:
            xy = (width - 2 - (p - (width + height - 1)), height - 1)
        else:
            xy = (0, height - 2 - (p - (2 * width + height - 2)))
        out.append(xy)
    return out


def flatten(design, width, height, io_locations=None, placed=None):
    """The placer's input for `design` on a width x height site grid.

    Movable cells: the logic cells in creation order (the order
    collect_movable_cells walks them), except those `placed` marks locked.
    Fixed cells: the IO pseudo-cells, at io_locations[name] or evenly along
    the perimeter, then the locked logic cells at their sites.  placed: name
    -> (x, y, locked); an unlocked entry pre-binds the cell (its initial
    site).  Nets: in creation order without the constant nets; pins: the
    driver (when it is a cell that remains) first, then the users.
    Returns (Netlist, Chip, info) where info maps movable / fixed indices
    back to cell names."""
    from .placer import Chip, Netlist

    placed = placed or {}
    cidx = {c.name: i for i, c in enumerate(design.cells)}
    const_cells = {cidx.get("$PACKER_GND"), cidx.get("$PACKER_VCC")}
    movable, fixed = [], []
    for i, c in enumerate(design.cells):
        if i in const_cells:
            continue
        if c.type in IO_TYPES:
            fixed.append(i)
        elif placed.get(c.name, (0, 0, False))[2]:
            fixed.append(i)
        else:
            movable.append(i)
    io = [i for i in fixed if design.cells[i].type in IO_TYPES]
    locked = [i for i in fixed if design.cells[i].type not in IO_TYPES]
    fixed = io + locked
    default_io = perimeter_sites(len(io), width, height)
    fx, fy, on_logic = [], [], []
    for k, i in enumerate(io):
        x, y = (io_locations or {}).get(design.cells[i].name, default_io[k])
        fx.append(x)
        fy.append(y)
        on_logic.append(0)
    for i in locked:
        x, y, _ = placed[design.cells[i].name]
        fx.append(x)
        fy.append(y)
        on_logic.append(1)
    pid = {}
    for k, i in enumerate(movable):
        pid[i] = k
    for k, i in enumerate(fixed):
        pid[i] = len(movable) + k
    off, pins, has_driver = [0], [], []
    for n in design.nets:
        if n.name in (GND_NET, VCC_NET):
            continue
        net_pins = []
        driven = n.driver is not None and n.driver[0] in pid
        if driven:
            net_pins.append(pid[n.driver[0]])
        net_pins += [pid[c] for c, _ in n.users if c in pid]
        pins += net_pins
        off.append(len(pins))
        has_driver.append(1 if driven else 0)
    init_x = init_y = None
    if any(design.cells[i].name in placed for i in movable):
        init_x = np.array([placed.get(design.cells[i].name, (-1, -1, False))[0] for i in movable], np.int32)
        init_y = np.array([placed.get(design.cells[i].name, (-1, -1, False))[1] for i in movable], np.int32)
    nl = Netlist(num_cells=len(movable), net_offsets=np.array(off, np.uint32), pin_cell=np.array(pins, np.uint32),
                 fixed_x=np.array(fx, np.int32), fixed_y=np.array(fy, np.int32),
                 fixed_on_logic=np.array(on_logic, np.uint8) if locked else None,
                 net_has_driver=np.array(has_driver, np.uint8), cell_init_x=init_x, cell_init_y=init_y)
    info = {"movable": [design.cells[i].name for i in movable], "fixed": [design.cells[i].name for i in fixed]}
    return nl, Chip(width, height), info


def load_yosys_json(path_or_text, width, height, **kw):
    """Parse (a path or the JSON text) and flatten in one step."""
    text = path_or_text
    if not path_or_text.lstrip().startswith("{"):
        with open(path_or_text) as f:
            text = f.read()
    return flatten(parse_yosys_json(text), width, height, **kw)
