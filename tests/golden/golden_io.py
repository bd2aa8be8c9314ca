"""Serialisation of scenarios and results for the golden fixtures."""
import json

import numpy as np

from pacific_b200 import scenarios as S

STATE_KEYS = ["position", "quaternion", "velocity", "omega"]
STATIC_KEYS = ["id", "shape", "material", "radius", "crust", "mass", "inertia"]


def scenario_to_npz_dict(sc, prefix="in_"):
    spec = dict(name=sc.name, shapes=sc.shapes, dt=sc.dt, n_steps=sc.n_steps,
                domains=[{k: (np.asarray(v).tolist() if k != "cell_size" else v) for k, v in d.items()}
                         for d in sc.domains],
                laws=[[list(l[:3]) + [list(l[3])] for l in ls] for ls in sc.laws],
                obstacles=[[{k: (list(v) if isinstance(v, (list, tuple, np.ndarray)) else v) for k, v in o.items()}
                            for o in obs] for obs in sc.obstacles])
    if sc.meta.get("collision") is not None:
        spec["collision"] = sc.meta["collision"]
    if sc.meta.get("loadings"):
        spec["loadings"] = [[{k: (list(v) if isinstance(v, (list, tuple, np.ndarray)) else v) for k, v in l.items()}
                             for l in ls] for ls in sc.meta["loadings"]]
    out = {"spec": np.array(json.dumps(spec))}
    for k in STATIC_KEYS + STATE_KEYS:
        out[prefix + k] = np.asarray(sc.particles[k])
    # the orientation matrix of non-spherical bodies: the reference composes it
    # with each step's rotation, so after many steps it is not the matrix of the
    # quaternion to the last bit
    if sc.particles.get("basis") is not None:
        out[prefix + "basis"] = np.asarray(sc.particles["basis"])
    return out


def scenario_from_npz(z, prefix="in_"):
    spec = json.loads(str(z["spec"]))
    p = {k: np.array(z[prefix + k]) for k in STATIC_KEYS + STATE_KEYS}
    p["system"] = None
    p["basis"] = np.array(z[prefix + "basis"]) if prefix + "basis" in z.files else None
    doms = [dict(origin=np.array(d["origin"]), size=np.array(d["size"]), cell_size=d["cell_size"],
                 gravity=tuple(d["gravity"])) for d in spec["domains"]]
    laws = [[(l[0], l[1], l[2], l[3]) for l in ls] for ls in spec["laws"]]
    sc = S.Scenario(spec["name"], [tuple(s) for s in spec["shapes"]], doms, laws, spec["obstacles"], p,
                    spec["dt"], spec["n_steps"])
    if spec.get("loadings"):
        sc.meta["loadings"] = spec["loadings"]
    if spec.get("collision") is not None:
        sc.meta["collision"] = spec["collision"]
    return sc


def memory_arrays(mem, prefix):
    return {prefix + k: np.asarray(v) for k, v in mem.items()}


def memory_from(z, prefix):
    return {k: np.array(z[prefix + k]) for k in ["owner", "other", "kdelta", "prev_normal", "spring_torque"]}
