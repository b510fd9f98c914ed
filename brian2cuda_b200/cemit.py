"""Generated host code: a lowered Program as a standalone C program that builds and runs
the network through include/b2b.h and writes the monitors' records to result files.

This is the role of the project brian2cuda generates (`templates/main.cu:49-104` main(),
`templates/objects.cu:185-726` arrays loaded from and written to files,
`templates/network.cu:40-137` the run loop, `templates/makefile:1-23`): here the generated
code is plain C (no kernels: they live in libb2b.so) and is compiled with the host compiler,
`cc -I include main.c -L<dir of libb2b.so> -lb2b`.  Arrays too large to write into the
source (initial values, explicit connectivity) go to `static_arrays/<k>.bin` beside it, as
raw little-endian values; results go to `results/<monitor>_<field>.bin` in the dtypes the
Python side reads (int32 indices, int64 steps, state values in the variable's dtype).
"""
from __future__ import annotations

import os
import subprocess

import numpy as np

from .lowering import Program, _Ref
from .network import HH, LIF, STDP

_VAR = {"v": "B2B_VAR_V", "ge": "B2B_VAR_GE", "gi": "B2B_VAR_GI", "m": "B2B_VAR_M",
        "h": "B2B_VAR_H", "n": "B2B_VAR_N", "lastspike": "B2B_VAR_LASTSPIKE",
        "not_refractory": "B2B_VAR_NOT_REFRACTORY"}
_DT = {"float32": "B2B_F32", "float64": "B2B_F64"}


def _lit(x: float) -> str:
    x = float(x)
    if np.isinf(x):
        return "INFINITY" if x > 0 else "(-INFINITY)"
    return repr(x)


class _Emitter:
    def __init__(self, prog: Program, outdir: str):
        self.p = prog
        self.dir = outdir
        self.lines: list[str] = []
        self.n_arrays = 0
        self.gdtype: dict = {}      # group key -> numpy dtype of its state
        self.gsize: dict = {}
        self.names: dict = {}       # key -> C identifier
        os.makedirs(os.path.join(outdir, "static_arrays"), exist_ok=True)

    def ident(self, key: str) -> str:
        if key not in self.names:
            self.names[key] = "id_" + "".join(c if c.isalnum() else "_" for c in key)
        return self.names[key]

    def array(self, a: np.ndarray, ctype: str) -> str:
        k = self.n_arrays
        self.n_arrays += 1
        path = os.path.join(self.dir, "static_arrays", f"{k}.bin")
        np.ascontiguousarray(a).tofile(path)
        var = f"arr{k}"
        self.lines.append(f"  {ctype}* {var} = ({ctype}*)load_array(\"{k}\", "
                          f"sizeof({ctype}) * (size_t){a.size});")
        self.lines.append(f"  if (!{var}) return 2;")
        return var

    def ref(self, a) -> str:
        return self.ident(a.key) if isinstance(a, _Ref) else str(a)

    def emit(self):
        L = self.lines
        for op in self.p.ops:
            m, a, kw = op.method, op.args, op.kwargs
            out = self.ident(op.key) if op.key else None
            if m in ("lif_group", "hh_group"):
                n, prm, dtype = a
                self.gdtype[op.key] = np.float32 if dtype == "float32" else np.float64
                self.gsize[op.key] = n
                if isinstance(prm, LIF):
                    L.append(f"  {{ b2b_lif_params p = {{{_lit(prm.El)}, {_lit(prm.taum)}, "
                             f"{_lit(prm.taue)}, {_lit(prm.taui)}, {_lit(prm.ke)}, "
                             f"{_lit(prm.ki)}, {_lit(prm.Vt)}, {_lit(prm.Vr)}, "
                             f"{_lit(prm.refractory)}, {int(prm.has_threshold)}, "
                             f"{int(prm.has_reset)}, {int(prm.unless_refractory)}, 0}};")
                    L.append(f"    CHECK(b2b_group_lif(net, {n}, {_DT[dtype]}, &p, &{out})); }}")
                else:
                    assert isinstance(prm, HH)
                    vals = ", ".join(_lit(x) for x in prm.as_array())
                    L.append(f"  {{ b2b_hh_params p = {{{vals}}};")
                    L.append(f"    CHECK(b2b_group_hh(net, {n}, {_DT[dtype]}, &p, &{out})); }}")
            elif m == "model_group":
                n, gm, dtype = a
                from .codegen import compile_model
                if gm.path is None:
                    gm.path = compile_model(gm.source)
                self.gdtype[op.key] = np.float32 if dtype == "float32" else np.float64
                self.gsize[op.key] = n
                path = gm.path.replace("\\", "\\\\").replace('"', '\\"')
                L.append(f"  CHECK(b2b_group_model(net, {n}, {_DT[dtype]}, \"{path}\", "
                         f"{_lit(gm.refractory)}, &{out}));")
            elif m == "poisson_group":
                n, rate, dtype = a
                self.gdtype[op.key] = np.float32 if dtype == "float32" else np.float64
                self.gsize[op.key] = n
                L.append(f"  CHECK(b2b_group_poisson(net, {n}, {_DT[dtype]}, {_lit(rate)}, "
                         f"&{out}));")
            elif m == "spikegen_group":
                n, idx, steps = a
                self.gdtype[op.key] = np.float32
                self.gsize[op.key] = n
                ai = self.array(np.asarray(idx, np.int32), "int32_t")
                at = self.array(np.asarray(steps, np.int64), "int64_t")
                L.append(f"  CHECK(b2b_group_spikegen(net, {n}, {len(idx)}, {ai}, {at}, "
                         f"&{out}));")
                if kw.get("period"):
                    L.append(f"  CHECK(b2b_spikegen_period(net, {out}, {int(kw['period'])}));")
            elif m == "set_state":
                g, var, vals = a
                dt = np.uint8 if var == "not_refractory" else self.gdtype[g.key]
                ctype = {np.uint8: "uint8_t", np.float32: "float", np.float64: "double"}[dt]
                arr = self.array(np.asarray(vals).astype(dt), ctype)
                L.append(f"  CHECK(b2b_state_set(net, {self.ref(g)}, {_VAR[var]}, {arr}, "
                         f"{len(vals)}));")
            elif m == "synapses_random":
                pre, post, tgt, p, dmin, dmax, w, seed = a
                lo, hi = kw["pre_range"]
                L.append(f"  CHECK(b2b_synapses_random(net, {self.ref(pre)}, {lo}, {hi}, "
                         f"{self.ref(post)}, {_VAR[tgt]}, {_lit(p)}, {dmin}, {dmax}, {_lit(w)}, "
                         f"{int(seed)}ULL, &{out}));")
            elif m == "synapses":
                pre, post, tgt, i, j = a
                ai = self.array(np.asarray(i, np.int32), "int32_t")
                aj = self.array(np.asarray(j, np.int32), "int32_t")
                wdt = self.gdtype[post.key]
                wa = "NULL"
                if kw.get("w") is not None:
                    wa = self.array(np.asarray(kw["w"]).astype(wdt),
                                    "float" if wdt == np.float32 else "double")
                d = kw.get("delay", 0)
                if np.ndim(d) == 0:
                    da, ds = "NULL", int(d)
                else:
                    da, ds = self.array(np.asarray(d, np.int32), "int32_t"), 0
                st = kw.get("stdp")
                eff = "B2B_EFFECT_ADD"
                sp = "NULL"
                if st is not None:
                    assert isinstance(st, STDP)
                    eff = "B2B_EFFECT_STDP"
                    L.append(f"  b2b_stdp_params stdp_{out} = {{{_lit(st.taupre)}, "
                             f"{_lit(st.taupost)}, {_lit(st.dApre)}, {_lit(st.dApost)}, "
                             f"{_lit(st.wmin)}, {_lit(st.wmax)}, {int(st.pre_adds_weight)}, 0}};")
                    sp = f"&stdp_{out}"
                L.append(f"  CHECK(b2b_synapses(net, {self.ref(pre)}, {self.ref(post)}, "
                         f"{_VAR[tgt]}, {eff}, {len(i)}, {ai}, {aj}, {wa}, "
                         f"{_lit(kw.get('w_scalar', 0.0))}, {da}, {ds}, {sp}, &{out}));")
            elif m == "spike_monitor":
                g, cap = a
                L.append(f"  CHECK(b2b_spikemon(net, {self.ref(g)}, {int(cap)}));")
            elif m == "state_monitor":
                g, var, idx = a
                ai = self.array(np.asarray(idx, np.int64), "int64_t")
                L.append(f"  CHECK(b2b_statemon(net, {self.ref(g)}, {_VAR[var]}, {ai}, "
                         f"{len(idx)}, {int(kw['every'])}, {int(kw['capacity'])}, &{out}));")
            elif m == "rate_monitor":
                (g,) = a
                L.append(f"  CHECK(b2b_ratemon(net, {self.ref(g)}, {int(kw['capacity'])}, "
                         f"&{out}));")
            elif m == "poisson_input":
                g, var, n, rate, w = a
                L.append(f"  CHECK(b2b_poisson_input(net, {self.ref(g)}, {_VAR[var]}, {n}, "
                         f"{_lit(rate)}, {_lit(w)}, &{out}));")
            else:
                raise NotImplementedError(f"no C form for {m}")

    def results(self):
        L = self.lines
        for name, m in self.p.monitors.items():
            nm = "".join(c if c.isalnum() else "_" for c in name)
            if m["kind"] == "spike":
                g = self.ident(m["group"])
                lo, hi = m["sub"] if m["sub"] else (0, self.gsize[m["group"]])
                L.append(f"  {{ int64_t n = 0;")
                L.append(f"    CHECK(b2b_spikemon_get_range(net, {g}, {lo}, {hi}, &n, NULL, "
                         f"NULL, 0));")
                L.append("    int32_t* idx = (int32_t*)malloc(sizeof(int32_t) * (n + 1));")
                L.append("    int64_t* st = (int64_t*)malloc(sizeof(int64_t) * (n + 1));")
                L.append(f"    CHECK(b2b_spikemon_get_range(net, {g}, {lo}, {hi}, &n, idx, st, "
                         f"n));")
                L.append(f"    write_result(\"{nm}_i\", idx, sizeof(int32_t) * n);")
                L.append(f"    write_result(\"{nm}_t\", st, sizeof(int64_t) * n);")
                L.append("    free(idx); free(st); }")
            elif m["kind"] == "rate":
                mid = self.ident(name)
                L.append(f"  {{ int64_t n = 0;")
                L.append(f"    CHECK(b2b_ratemon_get(net, {mid}, &n, NULL, NULL, 0));")
                L.append("    int64_t* st = (int64_t*)malloc(sizeof(int64_t) * (n + 1));")
                L.append("    int32_t* c = (int32_t*)malloc(sizeof(int32_t) * (n + 1));")
                L.append(f"    CHECK(b2b_ratemon_get(net, {mid}, &n, st, c, n));")
                L.append(f"    write_result(\"{nm}_t\", st, sizeof(int64_t) * n);")
                L.append(f"    write_result(\"{nm}_count\", c, sizeof(int32_t) * n);")
                L.append("    free(st); free(c); }")
            else:
                for v in m["vars"]:
                    mid = self.ident(f"{name}:{v}")
                    es = "sizeof(uint8_t)" if v == "not_refractory" else (
                        "sizeof(float)" if self.gdtype[m["group"]] == np.float32
                        else "sizeof(double)")
                    vn = "".join(c if c.isalnum() else "_" for c in v)
                    L.append(f"  {{ int64_t n = 0;")
                    L.append(f"    CHECK(b2b_statemon_get(net, {mid}, &n, NULL, NULL, 0));")
                    L.append(f"    int64_t width = {self._state_width(name, v)};")
                    L.append("    int64_t* st = (int64_t*)malloc(sizeof(int64_t) * (n + 1));")
                    L.append(f"    void* val = malloc({es} * (size_t)(n * width + 1));")
                    L.append(f"    CHECK(b2b_statemon_get(net, {mid}, &n, st, val, n));")
                    L.append(f"    write_result(\"{nm}_{vn}_t\", st, sizeof(int64_t) * n);")
                    L.append(f"    write_result(\"{nm}_{vn}\", val, {es} * (size_t)(n * width));")
                    L.append("    free(st); free(val); }")

    def _state_width(self, name, v):
        for op in self.p.ops:
            if op.method == "state_monitor" and op.key == f"{name}:{v}":
                return len(op.args[2])
        raise KeyError(name)

    def source(self) -> str:
        decl = "".join(f"static int32_t {c} = -1;\n" for c in self.names.values())
        body = "\n".join(self.lines)
        runs = "\n".join(f"  CHECK(b2b_run(net, {int(s)}));" for s in self.p.runs)
        return _TEMPLATE.format(dt=repr(self.p.dt), seed=int(self.p.seed), decl=decl,
                                body=body, runs=runs)


_TEMPLATE = r"""/* Generated by brian2cuda_b200.cemit: builds and runs the network through libb2b's C ABI
 * (include/b2b.h).  Usage: ./main [results_dir]; reads static_arrays/ beside the binary's
 * working directory. */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "b2b.h"

static b2b_net* net = NULL;
static const char* results_dir = "results";
{decl}
#define CHECK(call)                                                                   \
  do {{                                                                               \
    b2b_status s_ = (call);                                                           \
    if (s_ != B2B_OK) {{                                                              \
      char msg_[512] = "";                                                            \
      if (net) b2b_last_error(net, msg_, sizeof msg_);                                \
      fprintf(stderr, "%s failed: %s (%s)\n", #call, b2b_status_string(s_), msg_);   \
      return 1;                                                                       \
    }}                                                                                \
  }} while (0)

static inline void* load_array(const char* name, size_t bytes) {{
  char path[1024];
  snprintf(path, sizeof path, "static_arrays/%s.bin", name);
  FILE* f = fopen(path, "rb");
  if (!f) {{ fprintf(stderr, "cannot open %s\n", path); return NULL; }}
  void* p = malloc(bytes ? bytes : 1);
  size_t got = bytes ? fread(p, 1, bytes, f) : 0;
  fclose(f);
  if (got != bytes) {{ fprintf(stderr, "short read %s\n", path); free(p); return NULL; }}
  return p;
}}

static inline void write_result(const char* name, const void* data, size_t bytes) {{
  char path[1024];
  snprintf(path, sizeof path, "%s/%s.bin", results_dir, name);
  FILE* f = fopen(path, "wb");
  if (!f) {{ fprintf(stderr, "cannot write %s\n", path); return; }}
  if (bytes) fwrite(data, 1, bytes, f);
  fclose(f);
}}

static int build_and_run(void) {{
  b2b_config cfg;
  memset(&cfg, 0, sizeof cfg);
  cfg.dt = {dt};
  cfg.device = 0;
  cfg.steps_per_graph = 50;
  cfg.seed = {seed}ULL;
  CHECK(b2b_create(&cfg, &net));
{body}
  CHECK(b2b_finalize(net));
{runs}
  int32_t device_status = 0;
  CHECK(b2b_sync(net, &device_status));
  if (device_status != B2B_OK) {{
    fprintf(stderr, "device status %s\n", b2b_status_string(device_status));
    return 3;
  }}
  return -1;   /* results follow */
}}

int main(int argc, char** argv) {{
  if (argc > 1) results_dir = argv[1];
  int rc = build_and_run();
  if (rc >= 0) {{ if (net) b2b_destroy(net); return rc; }}
  rc = write_results();
  b2b_destroy(net);
  return rc;
}}
"""


def emit_c(prog: Program, outdir: str) -> str:
    """Writes main.c and static_arrays/ for `prog` into outdir; returns main.c's path."""
    em = _Emitter(prog, outdir)
    em.emit()
    build = em.source()
    em.lines = []
    em.results()
    res_fn = ("static int write_results(void) {\n" + "\n".join(em.lines) +
              "\n  return 0;\n}\n")
    src = build.replace("int main(int argc", res_fn + "\nint main(int argc", 1)
    src = src.replace("static int build_and_run(void)",
                      "static int write_results(void);\nstatic int build_and_run(void)", 1)
    path = os.path.join(outdir, "main.c")
    with open(path, "w") as f:
        f.write(src)
    return path


def compile_c(outdir: str, cc: str = "cc") -> str:
    """Compiles outdir/main.c against include/b2b.h and libb2b.so (rpath set to the
    library's directory); returns the executable's path."""
    from . import _native
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    libdir = os.path.dirname(_native.lib_path())
    exe = os.path.join(outdir, "main")
    cmd = [cc, "-O2", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(root, "include"),
           os.path.join(outdir, "main.c"), "-L", libdir, "-lb2b", f"-Wl,-rpath,{libdir}",
           "-lm", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"cc failed:\n{r.stdout}\n{r.stderr}")
    return exe


def read_results(prog: Program, results_dir: str) -> dict:
    """The result files of a run, in the form Program.execute returns."""
    out = {}

    def rd(name, dt):
        return np.fromfile(os.path.join(results_dir, name + ".bin"), dtype=dt)
    for name, m in prog.monitors.items():
        nm = "".join(c if c.isalnum() else "_" for c in name)
        if m["kind"] == "spike":
            out[name] = (rd(nm + "_i", np.int32), rd(nm + "_t", np.int64))
        elif m["kind"] == "rate":
            out[name] = (rd(nm + "_t", np.int64), rd(nm + "_count", np.int32))
        else:
            d = {}
            for v in m["vars"]:
                vn = "".join(c if c.isalnum() else "_" for c in v)
                st = rd(f"{nm}_{vn}_t", np.int64)
                op = [o for o in prog.ops if o.key == f"{name}:{v}"][0]
                width = len(op.args[2])
                dt = np.float32 if prog.groups[m["group"]].get("dtype") == "float32" \
                    else np.float64
                vals = rd(f"{nm}_{vn}", dt).reshape(len(st), width)
                d[v] = (st, vals)
            out[name] = d
    return out
