"""LoG checkpoints as the LoD scene that the kernels read.

* load_statedict         -- LoG/utils/command.py:12-16 (torch.load, unwrap 'state_dict')
* rebuild_ancestor_path  -- apps/ancestor.py:21-73 with the per-level torch loop replaced by one
                            device pass (fgs_ancestor_path); same table, same key handling, the
                            same IndexError where the reference raises
* tree_scene             -- the FilterGS view of a LoG model (apps/render.py:100-122,
                            FilterGS/filtergs.py:40-50): the raw gaussian.* parameters and the
                            tree.node_index / ancestor_path / tree / root_index buffers, on a device

State-dict keys follow LoG's modules: gaussian.{xyz, scaling (log), rotation (raw quaternion),
opacity (logit), colors (SH DC), shs (rest SH, [P, (d+1)^2 - 1, 3])} and tree.{root_index,
node_index, index_parent, local_index, depth, tree, ancestor_path | ancestor}
(LoG/model/level_of_gaussian.py:130-156, LoG/model/tensor_tree.py:5-20).
"""
import math

import torch

from ._lib import call
from .lod import TreeScene


def _p(t):
    import ctypes as C
    return None if t is None or t.numel() == 0 else C.c_void_p(t.data_ptr())


def _s():
    import ctypes as C
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def load_statedict(path, map_location="cpu"):
    """LoG/utils/command.py:12-16: a training checkpoint ({'state_dict': ..., ...}) or a bare state dict."""
    sd = torch.load(path, map_location=map_location, weights_only=False)
    if isinstance(sd, dict) and "state_dict" in sd:
        sd = sd["state_dict"]
    return sd


def ancestor_path_table(index_parent, depth, width, device=None):
    """The [P, width] ancestor table of a tree (int32, on a CUDA device): the device pass behind
    rebuild_ancestor_path.  Raises IndexError where apps/ancestor.py raises."""
    dev = torch.device(device) if device is not None else index_parent.device
    if dev.type != "cuda":
        raise ValueError("the ancestor_path builder runs on a CUDA device")
    par = index_parent.to(device=dev, dtype=torch.int32).contiguous()
    dep = depth.to(device=dev, dtype=torch.int32).contiguous()
    P = int(par.numel())
    if int(dep.numel()) != P:
        raise ValueError("tree.index_parent and tree.depth differ in length")
    L = int(width)
    out = torch.empty(P, L, dtype=torch.int32, device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    call("fgs_ancestor_path", P, _p(par), _p(dep), L, _p(out), _p(err), _s())
    if int(err.item()):
        raise IndexError("ancestor_path: a parent id is past the tree, or a depth is past the table width")
    return out


def rebuild_ancestor_path(state_dict, device="cuda"):
    """apps/ancestor.py:21-73: rebuild tree.ancestor_path from tree.index_parent and tree.depth.

    The width is that of the stored table (tree.ancestor_path, else tree.ancestor) or, without one,
    max(depth) + 1.  The new table (on `device`, the stored table's dtype) is written back under
    tree.ancestor_path, and under tree.ancestor when that key exists.  Returns (table, max_depth)."""
    for key in ("tree.index_parent", "tree.depth"):
        if key not in state_dict:
            raise KeyError(f"Missing '{key}' in checkpoint state_dict")
    index_parent, depth = state_dict["tree.index_parent"], state_dict["tree.depth"]
    ancestor_key = next((k for k in ("tree.ancestor_path", "tree.ancestor") if k in state_dict), None)
    P = int(depth.numel())
    if ancestor_key is not None:
        old = state_dict[ancestor_key]
        width, dtype = int(old.shape[1]), old.dtype
    else:
        width = int(depth.max().item()) + 1 if P > 0 else 1
        dtype = torch.int32
    if P == 0 or width == 0:
        table = torch.full((P, width), -1, dtype=dtype, device=device)
        max_depth = 0
    else:
        max_depth = int(depth.max().item())
        table = ancestor_path_table(index_parent, depth, width, device).to(dtype)
    state_dict["tree.ancestor_path"] = table
    if "tree.ancestor" in state_dict:
        state_dict["tree.ancestor"] = table
    return table, max_depth


def sh_degree_of(shs):
    """Degree of a rest-SH block [P, (d+1)^2 - 1, 3] (0 without one)."""
    if shs is None or shs.dim() < 2 or shs.shape[1] == 0:
        return 0
    d = int(round(math.sqrt(shs.shape[1] + 1))) - 1
    if (d + 1) ** 2 - 1 != shs.shape[1]:
        raise ValueError(f"gaussian.shs has {shs.shape[1]} coefficients, not (d+1)^2 - 1 for any degree d")
    return d


def tree_scene(state_dict, device="cuda", sh_degree=None, rebuild_ancestors=None):
    """TreeScene of a LoG state dict.

    rebuild_ancestors: None rebuilds the ancestor table only when the checkpoint has none, True
    always rebuilds it (apps/ancestor.py's job), False requires a stored one.  sh_degree: the
    degree used for colours (FilterGS's active_sh_degree); default the stored block's degree."""
    g = lambda k: state_dict[f"gaussian.{k}"]  # noqa: E731
    missing = [k for k in ("gaussian.xyz", "gaussian.scaling", "gaussian.rotation", "gaussian.opacity",
                           "gaussian.colors", "tree.node_index", "tree.tree", "tree.root_index")
               if k not in state_dict]
    if missing:
        raise KeyError(f"Missing {missing} in checkpoint state_dict")
    shs = state_dict.get("gaussian.shs")
    deg = sh_degree_of(shs) if sh_degree is None else int(sh_degree)
    if shs is not None and deg > sh_degree_of(shs):
        raise ValueError(f"sh_degree {deg} exceeds the stored SH block's degree {sh_degree_of(shs)}")
    stored = next((k for k in ("tree.ancestor_path", "tree.ancestor") if k in state_dict), None)
    if rebuild_ancestors or (rebuild_ancestors is None and stored is None):
        anc, _ = rebuild_ancestor_path(state_dict, device=device)
    elif stored is None:
        raise KeyError("the checkpoint has no tree.ancestor_path (pass rebuild_ancestors=True)")
    else:
        anc = state_dict[stored]
    return TreeScene(g("xyz"), g("scaling"), g("rotation"), g("opacity"), g("colors"),
                     shs if deg > 0 else None, state_dict["tree.node_index"], anc, state_dict["tree.tree"],
                     state_dict["tree.root_index"], sh_degree=deg if deg > 0 else 1, device=device)
