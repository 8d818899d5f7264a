"""The Fortran ISO_C_BINDING module (fortran/pci_gpu_mod.f90) against the C
headers: every pci_gpu_* entry a Fortran pconf host calls has an interface
of the same name and argument count (no Fortran compiler here, so names and
arities are what can be checked).  Left to C / Python hosts, by design: the
no-alloc J_av (device pointers and a CUDA stream), the learned correction's
training API (harvest, models) and the file-format, batch and MLP APIs,
whose counterparts a Fortran pconf already has or does not use."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NOT_FOR_FORTRAN = {"pci_gpu_j_av_noalloc", "pci_gpu_davidson_harvest", "pci_gpu_set_correction_model"}


def _c_decls():
    hdr = open(os.path.join(ROOT, "include", "pci_gpu.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    out = {}
    for m in re.finditer(r"^\s*(?:const\s+char\s*\*|int32_t|int64_t|int|void)\s*\*?\s*(pci_gpu_\w+)\s*\(([^)]*)\)\s*;",
                         hdr, re.M | re.S):
        args = [a for a in m.group(2).split(",") if a.strip() and a.strip() != "void"]
        out[m.group(1)] = len(args)
    return out


def _f90_decls():
    src = open(os.path.join(ROOT, "fortran", "pci_gpu_mod.f90")).read()
    src = re.sub(r"&\s*\n\s*", " ", src)                    # join continuation lines
    out = {}
    for m in re.finditer(r"(?:function|subroutine)\s+(pci_\w+)\s*\(([^)]*)\)\s*(?:&\s*)?bind\(C", src, re.I):
        args = [a for a in m.group(2).split(",") if a.strip()]
        out[m.group(1)] = len(args)
    return out


def test_fortran_module_binds_the_pconf_entry_points():
    c, f = _c_decls(), _f90_decls()
    assert len(c) >= 30
    missing = sorted(set(c) - set(f) - NOT_FOR_FORTRAN)
    assert not missing, missing
    for name, n in f.items():
        if name in c:
            assert n == c[name], (name, n, c[name])
