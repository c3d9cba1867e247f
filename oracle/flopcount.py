"""Count the algorithmic FP64 work of one network rhs evaluation.

Measurement infrastructure (not the product): builds a counting copy of a
generated network header -- every ``double`` replaced by a value type whose
arithmetic operators and math functions increment counters -- and evaluates
the rhs the kernels evaluate (rates_fixed + rates_var + mass-action rhs +
thermal equation) and the stoichiometric Jacobian on a seeded sample of
benchmark states, averaging over the sample (the piecewise rates branch on
the temperature).

Counting rules (the roofline's work figure): add, sub, mul, div, sqrt = 1
flop; exp, log, log10, pow, tanh = 1 each and also tallied separately as
special functions; min / max / fabs / comparisons = 0. Results go to
``oracle/_build/flops_<net>.json`` and, as the benchmark's work figures, to
``krome_x_b200/networks/net_<net>.flops.json``;
``python oracle/flopcount.py [net...]``.
"""
import json
import re
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
OUT = HERE / "_build"

COUNTER = r'''
#include <cmath>
#include <cstdio>
namespace kbfc {
struct Cnt { long flops = 0, special = 0; };
inline Cnt& cnt() { static Cnt c; return c; }
struct cd {
  double v;
  constexpr cd() : v(0.0) {}
  constexpr cd(double x) : v(x) {}
  explicit operator double() const { return v; }
  cd& operator+=(cd o) { ++cnt().flops; v += o.v; return *this; }
  cd& operator-=(cd o) { ++cnt().flops; v -= o.v; return *this; }
  cd& operator*=(cd o) { ++cnt().flops; v *= o.v; return *this; }
  cd& operator/=(cd o) { ++cnt().flops; v /= o.v; return *this; }
};
#define KBFC_BIN(op) \
  inline cd operator op(cd a, cd b) { ++cnt().flops; return cd(a.v op b.v); } \
  inline cd operator op(cd a, double b) { ++cnt().flops; return cd(a.v op b); } \
  inline cd operator op(double a, cd b) { ++cnt().flops; return cd(a op b.v); } \
  inline cd operator op(cd a, int b) { ++cnt().flops; return cd(a.v op b); } \
  inline cd operator op(int a, cd b) { ++cnt().flops; return cd(a op b.v); }
KBFC_BIN(+) KBFC_BIN(-) KBFC_BIN(*) KBFC_BIN(/)
inline cd operator-(cd a) { return cd(-a.v); }
#define KBFC_CMP(op) \
  inline bool operator op(cd a, cd b) { return a.v op b.v; } \
  inline bool operator op(cd a, double b) { return a.v op b; } \
  inline bool operator op(double a, cd b) { return a op b.v; } \
  inline bool operator op(cd a, int b) { return a.v op b; }
KBFC_CMP(<) KBFC_CMP(>) KBFC_CMP(<=) KBFC_CMP(>=) KBFC_CMP(==) KBFC_CMP(!=)
inline cd exp(cd a) { ++cnt().flops; ++cnt().special; return cd(std::exp(a.v)); }
inline cd log(cd a) { ++cnt().flops; ++cnt().special; return cd(std::log(a.v)); }
inline cd log10(cd a) { ++cnt().flops; ++cnt().special; return cd(std::log10(a.v)); }
inline cd tanh(cd a) { ++cnt().flops; ++cnt().special; return cd(std::tanh(a.v)); }
inline cd pow(cd a, cd b) { ++cnt().flops; ++cnt().special; return cd(std::pow(a.v, b.v)); }
inline cd exp10(cd a) { ++cnt().flops; ++cnt().special; return cd(std::pow(10.0, a.v)); }
inline cd sqrt(cd a) { ++cnt().flops; return cd(std::sqrt(a.v)); }
inline cd fabs(cd a) { return cd(std::fabs(a.v)); }
inline cd fmin(cd a, cd b) { return cd(std::fmin(a.v, b.v)); }
inline cd fmax(cd a, cd b) { return cd(std::fmax(a.v, b.v)); }
inline bool isfinite(cd a) { return std::isfinite(a.v); }
}  // namespace kbfc
'''

DRIVER = r'''
int main(int argc, char** argv) {
  using namespace kbnet;
  const int nsample = %(ns)d;
  static const double Y[%(ns)d][%(neq)d] = %(ys)s;
  static const double PAR[%(ns)d][NPAR] = %(ps)s;
  long f_rhs = 0, s_rhs = 0, f_jac = 0, s_jac = 0;
  for (int c = 0; c < nsample; ++c) {
    kbfc::cd y[%(neq)d], f[%(neq)d], k[NREA + 1], J[NSPEC * NSPEC];
    for (int i = 0; i < %(neq)d; ++i) y[i] = Y[c][i];
    Params p;
    kbfc::cd row[NPAR];
    for (int i = 0; i < NPAR; ++i) row[i] = PAR[c][i];
    params_from_row(row, p);
    kbfc::cnt() = kbfc::Cnt();
    const kbfc::cd T = kbfc::fmin(kbfc::fmax(y[NSPEC], p.Tcmb), 1e9);
    for (int i = 0; i <= NREA; ++i) k[i] = 0.0;
    rates_fixed(T, y, p, k);
    rates_var(T, y, p, k);
    rhs(y, k, f);
    f[NSPEC] = thermal_dTdt(kbfc::fmin(kbfc::fmax(y[NSPEC], 2.73), 1e9), y, k, p);
    f_rhs += kbfc::cnt().flops; s_rhs += kbfc::cnt().special;
    kbfc::cnt() = kbfc::Cnt();
    jac_stoich(y, k, J, NSPEC, 1);
    f_jac += kbfc::cnt().flops; s_jac += kbfc::cnt().special;
  }
  std::printf("{\"rhs_flops\": %%.3f, \"rhs_special\": %%.3f, \"jac_stoich_flops\": %%.3f}\n",
              (double)f_rhs / nsample, (double)s_rhs / nsample,
              (double)f_jac / nsample);
  return 0;
}
'''


def counting_source(key):
    """the network header and the physics it includes, with `double` and
    the math functions routed through the counting type"""
    def conv(text):
        text = re.sub(r"#include \"../csrc/kb_common.h\"", "", text)
        text = re.sub(r"#include \"../csrc/kb_conserve.h\"", "", text)
        text = re.sub(r"#include \"../csrc/kb_jacdk.h\"",
                      lambda m: conv((ROOT / "krome_x_b200/csrc/kb_jacdk.h")
                                     .read_text().replace("#pragma once", "")),
                      text)
        text = re.sub(r"#include \"../csrc/kb_physics.h\"",
                      lambda m: conv((ROOT / "krome_x_b200/csrc/kb_physics.h")
                                     .read_text()), text)
        text = re.sub(r"\bkb_exp10\(", "kbfc::exp10(", text)
        text = re.sub(r"\bkb_(exp|log10|log|pow)\(", r"kbfc::\1(", text)
        text = re.sub(r"\bdouble\b", "kbfc::cd", text)
        text = text.replace("std::", "kbfc::")
        text = re.sub(r"(?<![\w:])(isfinite|fmin|fmax|fabs|exp|log|log10|pow|sqrt|tanh)\(",
                      r"kbfc::\1(", text)
        return text
    common = (ROOT / "krome_x_b200/csrc/kb_common.h").read_text()
    common = common.replace("#pragma once", "")
    common = re.sub(r"template <int N>\s*KB_HD inline double ipow_\(double x\)",
                    "template <int N> KB_HD inline kbfc::cd ipow_(kbfc::cd x)",
                    common)
    common = common.replace("const double h = ipow_<N / 2>(x);",
                            "const kbfc::cd h = ipow_<N / 2>(x);")
    net = (ROOT / "krome_x_b200/networks" / ("net_%s.h" % key)).read_text()
    return COUNTER + common + conv(net)


def count(key, nsample=64):
    sys.path.insert(0, str(ROOT))
    from krome_x_b200 import netinfo, workloads
    info = netinfo.load(key)
    n, T, dt, par = workloads.GENERATORS[key](nsample, info, seed=31)
    y = np.concatenate([n, T[:, None]], axis=1)
    fmt = lambda a: "{" + ",".join("{" + ",".join(repr(float(v)) for v in r)
                                   + "}" for r in a) + "}"
    src = counting_source(key) + DRIVER % dict(
        ns=nsample, neq=y.shape[1], ys=fmt(y), ps=fmt(np.nan_to_num(par)))
    OUT.mkdir(parents=True, exist_ok=True)
    cpp = OUT / ("flopcount_%s.cpp" % key)
    exe = OUT / ("flopcount_%s" % key)
    cpp.write_text(src)
    subprocess.run(["g++", "-O1", "-std=c++17", "-w", str(cpp), "-o", str(exe)],
                   check=True)
    res = json.loads(subprocess.run([str(exe)], check=True, capture_output=True,
                                    text=True).stdout)
    res["network"] = key
    (OUT / ("flops_%s.json" % key)).write_text(json.dumps(res) + "\n")
    # the work figures the benchmark's roofline reads
    (ROOT / "krome_x_b200" / "networks" / ("net_%s.flops.json" % key)).write_text(
        json.dumps(res, indent=1) + "\n")
    return res


if __name__ == "__main__":
    for k in sys.argv[1:] or ["primordial", "primordial3", "galaxy_ism"]:
        print(count(k))
