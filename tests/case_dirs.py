"""Writes sonicSolver-format case directories for the host driver tests.

The files follow the layout and keys the reference's case directories use
(case.yaml; solvers/{solvers,runtime,numerics,algorithm}.yaml;
models/{models,thermoDynamics}.yaml; mesh/{mesh,generation}.yaml with a JSON
generation file; fields/{fields,internalField,boundaries}.yaml), filled from
the parameters given here.
"""
from __future__ import annotations

import json
import os


def _w(path, text):
    os.makedirs(os.path.dirname(path), exist_ok=True)
    with open(path, "w") as f:
        f.write(text)


def write_case(root, name, *, cells, box_hi, box_lo=(0.0, 0.0, 0.0), n_ghost=3, convection="weno5Rusanov",
               time="SSPRK3", end_time=0.2, cfl=0.5, write_interval=0.05, write_initial=False, gamma=1.4,
               left=(1.0, 0.0, 1.0), right=(0.125, 0.0, 0.1), boundaries=None, numerics_form="terms",
               vertices=None, hex=tuple(range(8)), grading=(1.0, 1.0, 1.0), edges=(), scale=1.0):
    """A Riemann problem: leftHalf / rightHalf states (rho, u, p) split at
    i < nx/2.  `boundaries` maps patch -> condition, or patch -> {field:
    condition} for per-field laws (written verbatim, so the SonicFile form
    `fixedValue: [1 0 0]` works); omitted patches get none.  Defaults to
    zeroGradient Left/Right and empty side patches.  The block is the box
    box_lo..box_hi unless `vertices` (with the block's `hex` of vertex
    indices) is given; `grading` per axis and arc `edges` ((v0, v1, point)
    each) go to the generation file as the reference's generator reads
    them."""
    if boundaries is None:
        boundaries = {"Left": "zeroGradient", "Right": "zeroGradient", "sideWalls": "empty", "frontBack": "empty"}
    d = os.path.join(root, name)
    _w(os.path.join(d, "case.yaml"),
       f"# Case identity.\nSonicFile:\n  object: case\n  type: registry\nformatVersion: 1\nname: {name}\n")
    _w(os.path.join(d, "solvers", "solvers.yaml"),
       "SonicFile:\n  object: solver\n  type: registry\n"
       "runtime:\n  type: runtime\n  file: solvers/runtime.yaml\n"
       "numerics:\n  type: numerics\n  file: solvers/numerics.yaml\n"
       "algorithm:\n  type: algorithm\n  file: solvers/algorithm.yaml\n")
    _w(os.path.join(d, "solvers", "runtime.yaml"),
       "SonicFile:\n  object: solver\n  type: runtime\n"
       f"startTime: 0\nendTime: {end_time!r}\nCFL: {cfl!r}\nwriteControl: runTime\n"
       f"writeInterval: {write_interval!r}\nwriteInitial: {'true' if write_initial else 'false'}\n"
       f"output:\n  jobName: {name}\n  outputDir: result\n"
       "parallel:\n  enabled: false\n  nProcs: 1\n  split: [1, 1, 1]\n")
    if numerics_form == "terms":
        num = f"time:\n  default: {time}\nterms:\n  convection: {convection}\n"
    else:  # scheme / flux form
        scheme, flux = convection[:5], convection[5:]
        num = (f"time:\n  default: {time}\nconvection:\n  default: {scheme.upper()}\n"
               f"  formulation: conservativeFluxDifference\n  reconstruction: characteristic\n  flux: {flux}\n"
               "diffusion:\n  default: CENTRAL2\ntransport:\n  type: CENTRAL2\n  enable: false\n  mu: 0.0\n")
    _w(os.path.join(d, "solvers", "numerics.yaml"), "# Numerical methods.\nSonicFile:\n  object: solver\n"
       "  type: numerics\n" + num)
    _w(os.path.join(d, "solvers", "algorithm.yaml"), "SonicFile:\n  object: solver\n  type: algorithm\n"
       "type: densityBase\n")
    _w(os.path.join(d, "models", "models.yaml"), "SonicFile:\n  object: models\n  type: registry\n"
       "thermoDynamics:\n  type: thermoDynamics\n  file: models/thermoDynamics.yaml\n")
    _w(os.path.join(d, "models", "thermoDynamics.yaml"),
       "SonicFile:\n  object: models\n  type: thermoDynamics\nthermoDynamics:\n  equationOfState: perfectGas\n"
       f"  thermo: hConst\n  transport: const\nproperties:\n  equationOfState:\n    gamma: {gamma!r}\n"
       "    R: 287.05\n  transport:\n    mu: 0.0\n    Pr: 0.72\n")
    _w(os.path.join(d, "mesh", "mesh.yaml"), "SonicFile:\n  object: mesh\n  type: registry\n"
       "generation:\n  type: structuredMesh\n  file: mesh/generation.yaml\n")
    (x0, y0, z0), (x1, y1, z1) = box_lo, box_hi
    if vertices is None:
        vertices = [[x0, y0, z0], [x1, y0, z0], [x1, y1, z0], [x0, y1, z0],
                    [x0, y0, z1], [x1, y0, z1], [x1, y1, z1], [x0, y1, z1]]
    gen = {"SonicFile": {"object": "mesh", "type": "generation"}, "scale": float(scale), "nGhost": n_ghost,
           "vertices": [[float(c) for c in v] for v in vertices],
           "blocks": [{"vertices": [int(i) for i in hex], "cells": [int(c) for c in cells],
                       "grading": [float(g) for g in grading]}],
           "edges": [{"type": "arc", "vertices": [int(a), int(b)], "point": [float(c) for c in pt]}
                     for a, b, pt in edges],
           "patches": []}
    _w(os.path.join(d, "mesh", "generation.yaml"), json.dumps(gen, indent=2) + "\n")
    _w(os.path.join(d, "fields", "fields.yaml"), "SonicFile:\n  object: fields\n  type: registry\n"
       "internalField:\n  type: internalField\n  file: fields/internalField.yaml\n"
       "boundaries:\n  type: boundary\n  file: fields/boundaries.yaml\n")
    (rl, ul, pl), (rr, ur, pr) = left, right
    _w(os.path.join(d, "fields", "internalField.yaml"),
       "# Initial field values.\nSonicFile:\n  object: fields\n  type: internalField\n"
       f"U:\n  default: [0, 0, 0]\n  leftHalf: [{ul!r}, 0, 0]\n  rightHalf: [{ur!r}, 0, 0]\n"
       f"p:\n  default: 0\n  leftHalf: {pl!r}\n  rightHalf: {pr!r}\n"
       f"rho:\n  default: 0\n  leftHalf: {rl!r}\n  rightHalf: {rr!r}\n")
    def cond_of(cond, var):
        return cond[var] if isinstance(cond, dict) else cond
    body = ""
    for v in ("U", "p", "rho"):
        lines = "".join(f"  {patch}: {cond_of(cond, v)}\n" for patch, cond in boundaries.items()
                        if not isinstance(cond, dict) or v in cond)
        body += f"{v}:\n{lines}"
    _w(os.path.join(d, "fields", "boundaries.yaml"), "SonicFile:\n  object: fields\n  type: boundaries\n" + body)
    return d
