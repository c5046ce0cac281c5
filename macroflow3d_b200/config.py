"""The `flow:` section of the pipeline YAML, with the reference's keys and strictness.

Mirrors FlowYamlConfig / parse_flow (src/io/config/Config.hpp:86-114,
src/io/config/ConfigYaml.cpp:130-229) and HeadSolveConfig::from_yaml
(src/physics/flow/solve_head.cuh:98-130): unknown keys are errors, BC faces may be named
west/east/south/north/bottom/top or xmin..zmax, `pin: {mode: auto|on|off}` or the legacy
`pin_first_cell: bool`.  Keys this library adds (all optional): precision
(fp64|fp32|bf16), flexible (auto|true|false), conv_norm (r0|b), use_graph (bool).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, List, Tuple

import yaml

DIRICHLET, NEUMANN, PERIODIC = 0, 1, 2
SOLVER_PCG_MG, SOLVER_MG, SOLVER_CG = 0, 1, 2
PIN_AUTO, PIN_ON, PIN_OFF = 0, 1, 2
PREC = {"fp64": 0, "fp32": 1, "bf16": 2}

REFERENCE_KEYS = {"solver", "mg_levels", "mg_pre_smooth", "mg_post_smooth", "mg_coarse_iters",
                  "mg_max_cycles", "cg_max_iter", "cg_rtol", "cg_check_every", "rtol",
                  "verify_velocity", "pin", "pin_first_cell", "bc"}
EXTENSION_KEYS = {"precision", "flexible", "conv_norm", "use_graph"}
FACES = (("west", "xmin"), ("east", "xmax"), ("south", "ymin"), ("north", "ymax"),
         ("bottom", "zmin"), ("top", "zmax"))


class ConfigError(ValueError):
    pass


@dataclass
class BCFace:
    type: int = DIRICHLET
    value: float = 0.0


@dataclass
class BCSpec:
    """BCSpec (src/core/BCSpec.hpp:36-88); default all faces Dirichlet 0."""
    faces: List[BCFace] = field(default_factory=lambda: [BCFace() for _ in range(6)])

    @property
    def types(self) -> Tuple[int, ...]:
        return tuple(f.type for f in self.faces)

    @property
    def values(self) -> Tuple[float, ...]:
        return tuple(f.value for f in self.faces)

    def validate(self) -> None:
        for a in range(3):
            p0 = self.faces[2 * a].type == PERIODIC
            p1 = self.faces[2 * a + 1].type == PERIODIC
            if p0 != p1:
                raise ConfigError("Periodic BC must be specified on both faces of an axis")
        for f in self.faces:
            if f.value != f.value or f.value in (float("inf"), float("-inf")):
                raise ConfigError("BC values must be finite")

    @staticmethod
    def darcy_x(h_west: float = 1.0, h_east: float = 0.0) -> "BCSpec":
        """h = h_west at x = 0, h = h_east at x = L, homogeneous Neumann elsewhere."""
        return BCSpec([BCFace(DIRICHLET, h_west), BCFace(DIRICHLET, h_east)] +
                      [BCFace(NEUMANN, 0.0) for _ in range(4)])


@dataclass
class FlowConfig:
    """FlowYamlConfig defaults (Config.hpp:86-114) plus this library's extensions."""
    solver: str = "mg"
    mg_levels: int = 4
    mg_pre_smooth: int = 2
    mg_post_smooth: int = 2
    mg_coarse_iters: int = 50
    mg_max_cycles: int = 20
    cg_max_iter: int = 1000
    cg_rtol: float = 1e-8
    cg_check_every: int = 10
    rtol: float = 1e-6
    verify_velocity: bool = False
    pin_mode: int = PIN_AUTO
    bc: BCSpec = field(default_factory=BCSpec)
    precision: str = "fp64"
    flexible: str = "auto"
    conv_norm: str = "r0"
    use_graph: bool = True


_BC_TYPES = {"dirichlet": DIRICHLET, "Dirichlet": DIRICHLET, "neumann": NEUMANN,
             "Neumann": NEUMANN, "periodic": PERIODIC, "Periodic": PERIODIC}


def _parse_face(node, name: str) -> BCFace:
    if node is None:
        return BCFace()
    if not isinstance(node, dict):
        raise ConfigError(f"flow.bc.{name} must be a map")
    t = node.get("type", "dirichlet")
    if t not in _BC_TYPES:
        raise ConfigError(f"Unknown BC type: {t}")
    ft = _BC_TYPES[t]
    if ft == PERIODIC:
        return BCFace(PERIODIC, 0.0)
    return BCFace(ft, float(node.get("value", 0.0)))


def parse_flow(node: Dict, defaults: FlowConfig | None = None) -> FlowConfig:
    """parse_flow (ConfigYaml.cpp:130-229): returns a FlowConfig or raises ConfigError
    listing every unknown key."""
    cfg = FlowConfig() if defaults is None else FlowConfig(**defaults.__dict__)
    if not node:
        return cfg
    if not isinstance(node, dict):
        raise ConfigError("flow must be a map")
    errs = [f"Unknown key 'flow.{k}'" for k in node if k not in REFERENCE_KEYS | EXTENSION_KEYS]
    if errs:
        raise ConfigError("; ".join(errs))
    for k in ("solver", "mg_levels", "mg_pre_smooth", "mg_post_smooth", "mg_coarse_iters",
              "mg_max_cycles", "cg_max_iter", "cg_check_every", "cg_rtol", "rtol",
              "verify_velocity", "precision", "flexible", "conv_norm", "use_graph"):
        if k in node:
            setattr(cfg, k, node[k])
    for k in ("mg_levels", "mg_pre_smooth", "mg_post_smooth", "mg_coarse_iters", "mg_max_cycles",
              "cg_max_iter", "cg_check_every"):
        setattr(cfg, k, int(getattr(cfg, k)))
    cfg.cg_rtol, cfg.rtol = float(cfg.cg_rtol), float(cfg.rtol)
    if "pin" in node:
        mode = (node["pin"] or {}).get("mode", "auto")
        cfg.pin_mode = {"on": PIN_ON, "off": PIN_OFF}.get(mode, PIN_AUTO)
    elif "pin_first_cell" in node:
        cfg.pin_mode = PIN_ON if bool(node["pin_first_cell"]) else PIN_OFF
    if "bc" in node:
        bcn = node["bc"] or {}
        faces = list(cfg.bc.faces)
        for f, (legacy, coord) in enumerate(FACES):
            if legacy in bcn:
                faces[f] = _parse_face(bcn[legacy], legacy)
            elif coord in bcn:
                faces[f] = _parse_face(bcn[coord], coord)
        cfg.bc = BCSpec(faces)
    if str(cfg.precision) not in PREC:
        raise ConfigError(f"flow.precision must be one of {sorted(PREC)}")
    if str(cfg.conv_norm) not in ("r0", "b"):
        raise ConfigError("flow.conv_norm must be r0 or b")
    validate_flow(cfg)
    return cfg


def validate_flow(cfg: FlowConfig) -> None:
    """The flow checks of ConfigValidator.hpp:82-99."""
    if cfg.solver not in ("mg", "cg", "mg_cg", "pcg_mg"):
        raise ConfigError("flow.solver must be one of mg, cg, mg_cg")
    if cfg.mg_levels < 1:
        raise ConfigError("flow.mg_levels must be >= 1")
    if cfg.cg_max_iter < 1 or cfg.cg_check_every < 1:
        raise ConfigError("flow.cg_max_iter and flow.cg_check_every must be >= 1")
    if not (cfg.cg_rtol > 0 and cfg.rtol > 0):
        raise ConfigError("flow tolerances must be positive")
    cfg.bc.validate()


def load_flow_yaml(text_or_path: str) -> FlowConfig:
    """Loads the `flow:` section of a pipeline YAML (a path or the YAML text itself)."""
    try:
        with open(text_or_path) as f:
            doc = yaml.safe_load(f)
    except (OSError, ValueError):
        doc = yaml.safe_load(text_or_path)
    if not isinstance(doc, dict):
        raise ConfigError("config must be a YAML map")
    return parse_flow(doc.get("flow"))
