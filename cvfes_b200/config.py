"""cfg-driven set-up, mirroring the reference's ``cvconfig.py`` over a ConfigObj file.

ConfigObj is not a dependency; :func:`parse` reads the subset of its INI dialect
the reference's ``cfg/*.cfg`` files use: ``key = value`` lines, ``#`` comments,
quoted strings, comma lists and nested ``[section]`` / ``[[sub]]`` / ``[[[...]]]``
headers.  Sections offer ConfigObj's ``as_int``/``as_float``/``as_bool`` and
``sections``.

The config classes keep the reference's attribute names (``cvconfig.py:17-219``)
and add two optional sections used only by this package:

* ``[gpu]``: ``precision`` (fp64 | fp32), ``state`` (auto | previous | velocity),
  ``semantics`` (cpu | opencl), ``use_graph``, ``graph_chunk``,
  ``norms_every``, ``watchdog``, ``device``;
* ``[synthetic]``: a structured tube wall mesh with GMRF material samples in
  place of the VTP files the reference reads (see :mod:`cvfes_b200.cases`).

``[solver] pressure_ramp`` (``cosine`` — the reference's RefreshContext — or
``linear``) selects the load schedule.
"""
from __future__ import annotations

import re
from typing import Any, List, Optional

_TRUE = {"1", "true", "yes", "on"}
_FALSE = {"0", "false", "no", "off"}


class Section(dict):
    """One ConfigObj section: a dict of values plus ordered sub-sections."""

    def __init__(self, name: str = "", parent: Optional["Section"] = None):
        super().__init__()
        self.name = name
        self.parent = parent
        self.sections: List[str] = []
        self.scalars: List[str] = []

    def as_int(self, key: str) -> int:
        return int(float(self[key])) if "." in str(self[key]) or "e" in str(self[key]).lower() \
            else int(self[key])

    def as_float(self, key: str) -> float:
        return float(self[key])

    def as_bool(self, key: str) -> bool:
        v = str(self[key]).strip().lower()
        if v in _TRUE:
            return True
        if v in _FALSE:
            return False
        raise ValueError(f"{key} = {self[key]!r} is not a boolean")

    def get_float(self, key: str, default: float) -> float:
        return float(self[key]) if key in self else default

    def get_int(self, key: str, default: int) -> int:
        return self.as_int(key) if key in self else default

    def get_bool(self, key: str, default: bool) -> bool:
        return self.as_bool(key) if key in self else default

    def get_str(self, key: str, default: Optional[str]) -> Optional[str]:
        return str(self[key]) if key in self else default


def _strip_comment(line: str) -> str:
    out, quote = [], None
    for ch in line:
        if quote:
            if ch == quote:
                quote = None
        elif ch in "'\"":
            quote = ch
        elif ch == "#":
            break
        out.append(ch)
    return "".join(out).strip()


def _parse_value(raw: str) -> Any:
    items, cur, quote, quoted_any = [], [], None, False
    for ch in raw:
        if quote:
            if ch == quote:
                quote = None
            else:
                cur.append(ch)
        elif ch in "'\"":
            quote, quoted_any = ch, True
        elif ch == ",":
            items.append("".join(cur).strip())
            cur = []
        else:
            cur.append(ch)
    if quote:
        raise ValueError(f"unterminated quote in {raw!r}")
    last = "".join(cur).strip()
    if items:
        if last:
            items.append(last)
        return items
    return last if quoted_any else last.strip()


_HEADER = re.compile(r"^(\[+)\s*(.*?)\s*(\]+)$")


def parse(text_or_path: str) -> Section:
    """Parse a ConfigObj-style file (path) or string (if it contains a newline)."""
    if "\n" in text_or_path or "=" in text_or_path:
        text = text_or_path
    else:
        with open(text_or_path) as f:
            text = f.read()
    root = Section("root")
    stack = [root]
    for lineno, line in enumerate(text.splitlines(), 1):
        s = _strip_comment(line)
        if not s:
            continue
        m = _HEADER.match(s)
        if m:
            depth = len(m.group(1))
            if depth != len(m.group(3)):
                raise ValueError(f"line {lineno}: unbalanced section brackets")
            if depth > len(stack):
                raise ValueError(f"line {lineno}: section nested too deep")
            parent = stack[depth - 1]
            sec = Section(m.group(2), parent)
            parent[sec.name] = sec
            parent.sections.append(sec.name)
            del stack[depth:]
            stack.append(sec)
            continue
        if "=" not in s:
            raise ValueError(f"line {lineno}: expected key = value")
        k, v = s.split("=", 1)
        key = k.strip().strip("'\"")
        stack[-1][key] = _parse_value(v.strip())
        stack[-1].scalars.append(key)
    return root


# ---------------------------------------------------------------------------- classes
class MeshConfig:
    """``cvconfig.py:34-50``: name, file_path, domain_id and faces."""

    def __init__(self, sec: Section):
        self.name = sec.get_str("name", None)
        self.file_path = sec.get("file_path")
        self.domainId = sec.get_int("domain_id", 0)
        self.faces = []
        if "faces" in sec:
            for name in sec["faces"].sections:
                if name.startswith("face"):
                    f = sec["faces"][name]
                    self.faces.append(type("FaceConfig", (), {"name": f.get("name"),
                                                              "file_path": f.get("file_path")})())
        self.nSmp = None
        self.regenerate_samples = False


def _get_prop(sec: Section, key: str):
    sub = sec[key]
    if "uniform_value" in sub:
        return sub.as_float("uniform_value")
    if "uniform_func" in sub:
        return sub["uniform_func"]
    if "file_name" in sub:
        return sub["file_name"]
    raise KeyError(f"no value for {key}")


class EquationConfig:
    """``cvconfig.py:104-146`` (solid keys; fluid keys are read but unused here)."""

    def __init__(self, sec: Section):
        self.name = sec["name"]
        if self.name == "fluid":
            self.dviscosity = sec.get_float("dynamic_viscosity", 0.04)
            self.density = sec.get_float("density", 1.06)
            self.f = sec.get_float("external_force", 0.0)
            return
        self.thickness = sec.as_float("thickness")
        self.density = sec.as_float("density")
        self.E = sec.as_float("Youngs Modulus")
        self.v = sec.as_float("Poissons Ratio")
        self.damp = sec.as_float("Damp")
        self.thicknessFilename = sec.get_str("thickness Filename", None)
        self.sigmaThickness = sec.get_float("thickness sigma", 0.0)
        self.rhoThickness = sec.get_float("thickness rho", 3.7)
        self.YoungsModulusFilename = sec.get_str("Youngs Modulus Filename", None)
        self.sigmaE = sec.get_float("Youngs Modulus sigma", 0.0)
        self.rhoE = sec.get_float("Youngs Modulus rho", 3.7)
        ini = sec.get("initial conditions")
        bdy = sec.get("boundary conditions")
        self.iniVelocity = _get_prop(ini, "velocity") if ini and "velocity" in ini else 0.0
        self.iniDisplacement = _get_prop(ini, "displacement") if ini and "displacement" in ini else 0.0
        self.bdyDisplacement = _get_prop(bdy, "displacement") if bdy and "displacement" in bdy else 0.0


class SolverConfig:
    """``cvconfig.py:149-173`` plus the load-schedule selector."""

    def __init__(self, sec: Section):
        self.method = sec.get_str("method", "transient GPU")
        self.time = sec.get_float("time", 0.0)
        self.dt = sec.as_float("dt")
        self.endtime = sec.as_float("endtime")
        self.tolerance = sec.get_float("tolerance", 0.01)
        self.rho_infinity = sec.get_float("rho_infinity", 0.2)
        self.imax = sec.get_int("imax", 20)
        self.ci = sec.get_float("ci", 3.0)
        self.dt_f = sec.get_float("dt_f", 0.01)
        self.update_interval = sec.get_int("stiffness_update_interval", 0)
        self.constant_pressure = sec.get_float("constant_pressure", 0.0)
        self.constant_T = sec.get_float("constant_T", 1.0)
        self.pressure_ramp = sec.get_str("pressure_ramp", "cosine")
        self.time_rounding = sec.get_int("time_rounding", 4)
        self.restart = sec.get_bool("restart", False)
        self.restartFilename = sec.get_str("restart_displacement_file", None)
        self.restartTimestep = sec.get_int("restart_timestep", 0)
        self.saveStressFilename = None
        self.saveResNum = 0
        self.exportBdyStressFilename = None
        self.useConstantStress = False
        self.nSmp = 1


class GPUConfig:
    """``[gpu]``: precision and execution options of the sm_100a solid step."""

    def __init__(self, sec: Optional[Section]):
        sec = sec if sec is not None else Section("gpu")
        prec = sec.get_str("precision", "fp64").lower()
        if prec not in ("fp64", "fp32"):
            raise ValueError("[gpu] precision must be fp64 or fp32")
        self.precision = 64 if prec == "fp64" else 32
        self.use_graph = sec.get_bool("use_graph", True)
        self.graph_chunk = sec.get_int("graph_chunk", 48)
        self.norms_every = sec.get_int("norms_every", 0)
        self.watchdog = sec.get_bool("watchdog", True)
        self.device = sec.get_int("device", -1)
        # second state buffer of the template step: previous (u_{n-1}, the reference's
        # pair of displacements), velocity (the increment u_n - u_{n-1}, kept in its
        # own buffer) or auto (velocity for the FP32 state, previous for FP64)
        self.state = sec.get_str("state", "auto").lower()
        if self.state not in ("auto", "previous", "velocity"):
            raise ValueError("[gpu] state must be auto, previous or velocity")
        # numerics of the step: cpu (SolidSolver, physicsSolver.py) or opencl (the
        # OpenCL class the drop-in replaces, physicsSolverSDampGPUs.py/.cl)
        self.semantics = sec.get_str("semantics", "cpu").lower()
        if self.semantics not in ("cpu", "opencl"):
            raise ValueError("[gpu] semantics must be cpu or opencl")


class CVConfig:
    """``cvconfig.py:176-219``."""

    def __init__(self, root: Section):
        self.ndim = root.get_int("dimensions", 3)
        self.nSmp = root.get_int("sample_num", 1)
        self.regenerate_samples = root.get_bool("regenerate_samples", False)
        self.name = root.get_str("name", "spCy")
        self.meshes = {}
        if "meshes" in root:
            for s in root["meshes"].sections:
                if s.startswith("mesh"):
                    mc = MeshConfig(root["meshes"][s])
                    self.meshes[mc.name] = mc
        self.equations = {}
        if "equations" in root:
            for s in root["equations"].sections:
                if s.startswith("equation"):
                    ec = EquationConfig(root["equations"][s])
                    self.equations[ec.name] = ec
        self.solver = SolverConfig(root["solver"])
        self.solver.saveStressFilename = root.get_str("save_stress_filename", "displacement.npz")
        self.solver.saveResNum = root.get_int("save_result_num", 0)
        self.solver.exportBdyStressFilename = root.get_str("export_stress_filename", None)
        self.solver.useConstantStress = root.get_bool("use_constant_stress", False)
        self.gpu = GPUConfig(root.get("gpu"))
        self.synthetic = root.get("synthetic")
        if "wall" in self.meshes:
            self.meshes["wall"].nSmp = self.nSmp
            self.meshes["wall"].regenerate_samples = self.regenerate_samples
        self.solver.nSmp = self.nSmp
        self.solver.gpu = self.gpu

    def set_samples(self, nSmp: int):
        """The ``-s`` override of ``cvfes.py:42-45``."""
        self.nSmp = nSmp
        if "wall" in self.meshes:
            self.meshes["wall"].nSmp = nSmp
        self.solver.nSmp = nSmp


def load(path: str, nSmp: Optional[int] = None) -> CVConfig:
    cfg = CVConfig(parse(path))
    if nSmp is not None:
        cfg.set_samples(nSmp)
    return cfg
