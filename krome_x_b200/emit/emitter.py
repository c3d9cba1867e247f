"""Network emitter: writes the per-network device header the B200 kernels
compile against (``krome_x_b200/networks/net_<key>.h``).

Frontend. The network language is the reference's ``.knet`` format; the
emitter parses and resolves a network with the reference generator's own
frontend (``kromex.knet.parse_network`` and the ``kromex.codegen.Codegen``
resolution: piecewise groups, rate classification, parameters) and renders
each rate and variable expression with ``Codegen.cexpr``, so every rate is
the same arithmetic expression as in a reference project (reference:
kromex/codegen.py:1618-1733). The frontend is needed only when a header is
(re)generated, on a machine that has the reference tree; the generated
headers are committed and nothing at build or run time imports it.

Backend (this project's). The header is one host/device (``KB_HD``) scalar
form of the network, laid out for a warp-per-cell integrator where the
scalar network math is SIMT-uniform across lanes (every lane of a cell's
warp evaluates it on its own state: the base state, or a perturbed one in a
difference-quotient Jacobian column):

* ``rates_fixed`` / ``rates_var``: the rate coefficients of Tgas and the
  parameters only, and the rest (densities, externs); piecewise groups with
  the reference's ``outside=asym`` selection (zero below the group, the
  temperature clamped above it; reference: kromex/codegen.py:8052-8114);
* ``rhs``: mass-action dn/dt with each species' terms accumulated in
  reaction order, reactants then products (reference: kromex/codegen.py:
  4289-4327), so the sums round as the reference's do;
* ``jac_stoich``: the stoichiometric Jacobian d dn_i / d n_j of the rates
  held fixed (reference: kromex/codegen.py:8366-8378, 5172-5210);
* ``thermal_dTdt``: (gamma - 1)(heat - cool)/(kB ntot) with the configured
  processes in the reference's term order (reference:
  runtime/core/solve_cell.hpp:305-429), the network-derived terms (H2
  formation heating, collisional dissociation cooling, recombination
  cooling, the EXACT adiabatic index) emitted by the rules the reference
  generator applies (kromex/codegen.py:4900-5000, 6857-6966, 3697-3819).
"""
import re
import math
import os
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent.parent
# the physical constants of csrc/kb_common.h the emitter folds into numbers
kbc_boltzmann_erg = 1.380649e-16
kbc_amu = 1.6605390666e-24
OUTDIR = PKG / "networks"

# the benchmark networks and their generation options (the reference
# Preprocessor's thermal section)
NETWORKS = {
    "primordial": dict(network="primordial", cooling=["ATOMIC", "H2"],
                       heating=["CHEM", "COMPRESS"]),
    "primordial3": dict(network="primordial3",
                        cooling=["H2", "CONT", "CHEM"],
                        heating=["COMPRESS", "CHEM"],
                        h2_opacity="RIPAMONTI", gamma="EXACT"),
    "galaxy_ism": dict(network="galaxy_ism", cooling=[], heating=[]),
    # one more of the reference's networks, default thermal options: the
    # primordial gas with carbon and oxygen chemistry (27 species)
    "primordialZ": dict(network="primordialZ", cooling=[], heating=[]),
    # the early-universe chemistry (H, D, He, their ions and molecules; 16
    # species) with its RECFAST recombination rates, default thermal options
    "earlyUniverse": dict(network="earlyUniverse", cooling=[], heating=[]),
    # config 3: the surface options of the reference's cloudSurface test are
    # required by Semenov.knet (its binding energies)
    "semenov": dict(options_toml="examples/tests/cloudSurface/options.toml",
                    network_file="networks/Semenov.knet"),
    # a second large network on the sparse path: the reference's gas-phase
    # dark-cloud chemistry (networks/cloud.knet, 452 species), default
    # thermal options
    "cloud": dict(network="cloud", cooling=[], heating=[]),
}
# networks above this many species take the sparse path (one warp per cell,
# the state in HBM, the static-pivot sparse LU)
LARGE_NSPEC = 32

# H2-chemistry energy ledger of thermal CHEM (reactants, products, eV,
# thermalized): formation heats by its exothermicity times the HM79
# thermalized fraction, collisional dissociation cools by 4.48 eV
# (reference: kromex/codegen.py:4929-4937)
CHEM_LEDGER = [
    (["H", "H", "H"], ["H", "H2"], "4.48", True),
    (["H", "H", "H2"], ["H2", "H2"], "4.48", True),
    (["H", "H-"], ["H2", "e-"], "3.53", True),
    (["H", "H2+"], ["H+", "H2"], "1.83", True),
    (["H", "H2"], ["H", "H", "H"], "-4.48", False),
    (["H2", "e-"], ["H", "H", "e-"], "-4.48", False),
    (["H2", "H2"], ["H", "H", "H2"], "-4.48", False),
]


_REFERENCE = None  # set by main()'s --reference


def _reference_root():
    """the reference tree, whose generator frontend parses the network:
    --reference PATH, or the KROME_REFERENCE environment variable"""
    ref = _REFERENCE or os.environ.get("KROME_REFERENCE")
    if not ref:
        raise RuntimeError("the emitter needs the reference tree: pass "
                           "--reference PATH or set KROME_REFERENCE")
    return Path(ref)


def _frontend(cfg):
    """the resolved network: the reference generator's parse + Codegen,
    configured as a reference project with these options would be"""
    ref = _reference_root()
    for p in (str(ref), str(ref / "kromex")):
        if p not in sys.path:
            sys.path.insert(0, p)
    from kromex import Preprocessor
    import codegen
    import knet
    if cfg.get("options_toml"):
        kp = Preprocessor.from_file(str(ref / cfg["options_toml"]))
        kp.project.network = str(ref / cfg["network_file"])
    else:
        kp = Preprocessor(network=cfg["network"])
        kp.thermal.cooling = cfg.get("cooling", [])
        kp.thermal.heating = cfg.get("heating", [])
        if cfg.get("h2_opacity"):
            kp.thermal.h2_opacity = cfg["h2_opacity"]
        if cfg.get("gamma"):
            kp.thermal.gamma = cfg["gamma"]
    _, args = kp._args("/tmp/kb_emit_unused")
    args.network_file = args.network_pos or args.network
    net = knet.parse_network(args.network_file)
    if net.errors:
        raise RuntimeError("; ".join(net.errors))
    gen = codegen.Codegen(
        net, outside=args.outside, secion=args.secondary_ionization.split(","),
        num2col=args.num2col, metal_cooling=args.metal_cooling.split(","),
        dust_tables=args.dust_tables, gas_total=args.gas_total,
        cooling=args.cooling.split(","), heating=args.heating.split(","),
        cooling_floor=args.cooling_floor, evolve_rad=args.evolve_rad,
        evolve_Td=args.evolve_Td, shielding=args.shielding, gamma=args.gamma,
        h2_opacity=args.h2_opacity, photo_induced=args.photo_induced,
        photoelectric=args.photoelectric, wd01=args.wd01,
        cmb_pumping=args.cmb_pumping, habing_shield=args.habing_dust_shielding,
        reactant_multiplicity=args.reactant_multiplicity,
        screening=args.screening, binding_energies=args.binding_energies,
        surface_nu=args.surface_nu,
        surface_competition=not args.no_surface_competition,
        surface_tunnelling=not args.no_surface_tunnelling,
        reactive_desorption=args.reactive_desorption,
        cr_desorption=args.cr_desorption, surface_bins=args.surface_bins,
        rtol=args.rtol, atol=args.atol, cool_files=[],
        cool_levels=args.cool_levels, evolve_dust=args.evolve_dust,
        custom_atol=args.custom_atol, custom_rtol=args.custom_rtol,
        cool_escape=args.cool_escape, rhs=args.rhs)
    gen.generate_files()  # completes the resolution (parameters, groups)
    return net, gen, codegen


class Emitter:
    def __init__(self, key, cfg):
        self.key = key
        self.cfg = cfg
        self.net, self.gen, self.cg = _frontend(cfg)
        self.species = sorted(self.net.species)
        self.idx = {s: i for i, s in enumerate(self.species)}
        self.lines = []
        self.hoisted = {}

    # -- helpers -----------------------------------------------------------

    def w(self, s=""):
        self.lines.append(s)

    def cid(self, s):
        return self.gen.cid(s)

    def cx(self, ast, tvar):
        g = self.gen
        g._hoisted = dict(self.hoisted)
        g._in_ratefn = False
        s = g.cexpr(ast, tvar)
        return s.replace("constants::", "kbc::")

    def num(self, v):
        return self.gen.cnum(v)

    def den(self, sp):
        return "n[IDX_%s]" % self.cid(sp)

    # -- sections ----------------------------------------------------------

    def emit_head(self):
        net, gen = self.net, self.gen
        ns = len(self.species)
        nr = len(net.reactions)
        w = self.w
        w("// Generated by krome_x_b200.emit from the network '%s' -- do not "
          "edit." % net.name)
        w("// One host/device (KB_HD) scalar form of the network: species,")
        w("// parameters, rate coefficients, mass-action rhs, stoichiometric")
        w("// Jacobian and the thermal equation (see krome_x_b200/emit/")
        w("// emitter.py for the layout and the reference rules it follows).")
        w("#pragma once")
        w('#include "../csrc/kb_common.h"')
        w("")
        w("namespace kbnet {")
        w("")
        w('constexpr const char* NETWORK_NAME = "%s";' % net.name)
        w('constexpr const char* NETWORK_KEY = "%s";' % self.key)
        w("constexpr int NSPEC = %d;" % ns)
        w("constexpr int NREA = %d;" % nr)
        # the rates that depend on the densities (directly, through ntot or
        # Hnuclei, or through an extern function): the reference's analytic
        # Jacobian adds their dk/dn terms (kromex/codegen.py:8462-8560),
        # which jac_stoich below does not
        ndep = 0
        for rx in net.reactions:
            if rx["rate"]["kind"] != "expr":
                continue
            deps = self.gen.rate_deps(rx["rate"]["ast"])
            if deps is None or deps[0] or deps[1]:
                ndep += 1
        w("constexpr int KB_RATE_NDEP = %d;" % ndep)
        # species a freeze directive can hold (the reference turns its
        # charge-invariant Newton correction off on such networks,
        # solve_cell.hpp:1631-1642)
        w("#define KB_NFREEZE %d"
          % sum(len(f["species"]) for f in net.freeze))
        for i, s in enumerate(self.species):
            w("constexpr int IDX_%s = %d;" % (self.cid(s), i))
        for s in self.species:
            w("#define KB_HAS_%s 1" % self.cid(s))
        for f in sorted(net.externs):
            w("#define KB_EXTERN_%s 1" % f)
        w("constexpr int IDX_ELECTRON = %d;" % self.idx.get("e-", -1))
        w("")
        names = ", ".join('"%s"' % s for s in self.species)
        w("inline const char* const species_names[NSPEC] = {%s};" % names)
        sp = net.species
        mass_amu = [sp[s]["mass_amu"] for s in self.species]
        # masses in grams as the reference writes them (mass_amu * amu)
        import constants as kc  # the reference's constant table
        mass_g = [m * kc.amu for m in mass_amu]
        charge = [sp[s]["charge"] for s in self.species]
        nH = [float(self.gen._natoms_H(s)) if hasattr(self.gen, "_natoms_H")
              else float((sp[s]["composition"] or {}).get("H", 0))
              for s in self.species]
        # the element composition (the reference's emit_composition,
        # kromex/codegen.py:3544-3567: elements in sorted order, an opaque
        # species all zero), for the post-solve conservation
        elems = sorted({e for x in self.species
                        for e in (sp[x]["composition"] or {})})
        comp = [str((sp[x]["composition"] or {}).get(e, 0)
                    if not sp[x]["opaque"] else 0)
                for x in self.species for e in elems] or ["0"]
        w("constexpr int NELEM = %d;" % len(elems))
        w("inline const char* const element_names[%d] = {%s};"
          % (max(len(elems), 1),
             ", ".join('"%s"' % e for e in elems) if elems else '""'))
        self.meta_elements = (elems, [[(sp[x]["composition"] or {}).get(e, 0)
                                       if not sp[x]["opaque"] else 0
                                       for e in elems] for x in self.species])
        tabs = (("double", "species_mass_g", [repr(float(m)) for m in mass_g]),
                ("int", "species_charge", [str(c) for c in charge]),
                ("double", "species_natoms_H", [repr(x) for x in nH]),
                ("int", "species_opaque", ["1" if sp[x]["opaque"] else "0"
                                           for x in self.species]))
        self.natoms_H = list(nH)
        for ty, name, vals in tabs:
            body = ", ".join(vals)
            if ns > LARGE_NSPEC:
                # a large network's tables live in global memory on the
                # device (a function-local array indexed at run time would
                # be rebuilt in local memory at every call)
                w("inline constexpr %s %s_t_[NSPEC] = {%s};" % (ty, name, body))
                w("#ifdef __CUDACC__")
                w("__device__ const %s d_%s_[NSPEC] = {%s};" % (ty, name, body))
                w("#endif")
                w("KB_HD inline %s %s(int i) {" % (ty, name))
                w("#ifdef __CUDA_ARCH__")
                w("  return d_%s_[i];" % name)
                w("#else")
                w("  return %s_t_[i];" % name)
                w("#endif")
                w("}")
            else:
                w("KB_HD inline %s %s(int i) {" % (ty, name))
                w("  constexpr %s t_[NSPEC] = {%s};" % (ty, body))
                w("  return t_[i];")
                w("}")
        # species_element(i, e): atoms of element e in species i
        body = ", ".join(comp)
        w("inline constexpr int species_elements_t_[%d] = {%s};" % (len(comp), body))
        w("#ifdef __CUDACC__")
        w("__device__ const int d_species_elements_[%d] = {%s};" % (len(comp), body))
        w("#endif")
        w("KB_HD inline int species_element(int i, int e) {")
        w("#ifdef __CUDA_ARCH__")
        w("  return d_species_elements_[i * NELEM + e];")
        w("#else")
        w("  return species_elements_t_[i * NELEM + e];")
        w("#endif")
        w("}")
        # summing helpers: sequential sums in species order (reference:
        # generated net_<name>_core.hpp ntot_ / Hnuclei_ / rho_)
        w("KB_HD inline double ntot_(const double* n) {")
        w("  double s = 0.0;")
        w("KB_UNROLL")
        w("  for (int i = 0; i < NSPEC; ++i) s += n[i];")
        w("  return s;")
        w("}")
        w("KB_HD inline double Hnuclei_(const double* n) {")
        w("  double s = 0.0;")
        w("KB_UNROLL")
        w("  for (int i = 0; i < NSPEC; ++i) s += n[i] * species_natoms_H(i);")
        w("  return s;")
        w("}")
        w("KB_HD inline double rho_(const double* n) {")
        w("  double s = 0.0;")
        w("KB_UNROLL")
        w("  for (int i = 0; i < NSPEC; ++i) s += n[i] * species_mass_g(i);")
        w("  return s;")
        w("}")
        w("")
        # parameters
        univ = {nm: (dv, cm) for nm, dv, cm in self.cg.UNIVERSAL_PARAMS}
        pn = list(gen.pnames)
        req = set(gen.param_required)
        dflt = []
        for s in pn:
            if s in net.params:
                dflt.append(float(net.params[s]))
            else:
                dv = univ[s][0]
                dflt.append(None if dv is None else float(dv))
        # the photo reactions: their rates come from the cell's photon
        # field, integrated once per solve into Params::kph (0 without one)
        self.photo_rx = [rx for rx in net.reactions
                         if rx["rate"]["kind"] == "photo"]
        nph = len(self.photo_rx)
        w("constexpr int NPAR = %d;" % len(pn))
        w("constexpr int NPHOTO = %d;" % nph)
        w("struct Params {")
        for s in pn:
            w("  double %s;" % s)
        if nph:
            w("  // the photo rates sum_b sigma_rb Phi_b of the cell's field")
            w("  double kph[NPHOTO];")
        w("};")
        w("inline const char* const param_names[NPAR] = {%s};"
          % ", ".join('"%s"' % s for s in pn))
        w("// the defaults of a parameter row; NaN marks a REQUIRED parameter")
        w("inline double param_default(int i) {")
        w("  const double t_[NPAR] = {%s};" % ", ".join(
            "NAN" if d is None else repr(d) for d in dflt))
        w("  return t_[i];")
        w("}")
        w("inline const char* const param_required_by[NPAR] = {%s};" % ", ".join(
            '"%s"' % (gen.param_required_by.get(s, "") if s in req else "")
            .replace('"', "'") for s in pn))
        w("KB_HD inline void params_from_row(const double* row, Params& p) {")
        for i, s in enumerate(pn):
            w("  p.%s = row[%d];" % (s, i))
        for j in range(nph):
            w("  p.kph[%d] = 0.0;" % j)
        w("}")
        w("KB_HD inline int params_missing(const Params& p) {")
        w("  (void)p;")
        for i, s in enumerate(pn):
            if s in req:
                w("  if (p.%s != p.%s) return %d;" % (s, s, i))
        w("  return -1;")
        w("}")
        if net.freeze:
            # whether a freeze directive holds for this parameter row (its
            # condition uses parameters only, fixed during a call)
            w("KB_HD inline bool freeze_active(const Params& p) {")
            w("  (void)p;")
            for f in net.freeze:
                cond = "true" if f["cond"] is None else self.gen.cexpr(f["cond"])
                w("  if (%s) return true;  // knet line %d" % (cond, f["line"]))
            w("  return false;")
            w("}")
            # the species held while their directive's condition holds:
            # their rows of the rhs and the Jacobian are zero and they do
            # not move in the conservation (the reference's generated
            # frozen_species, used at solve_cell.hpp:711-720, 1118-1131,
            # 1442-1450)
            w("KB_HD inline int frozen_species(const Params& p, int* idx) {")
            w("  (void)p; (void)idx;")
            w("  int m = 0;")
            for f in net.freeze:
                rows = " ".join("idx[m++] = IDX_%s;" % self.cid(sp)
                                for sp in f["species"])
                if f["cond"] is None:
                    w("  %s  // knet line %d" % (rows, f["line"]))
                else:
                    w("  if (%s) {  // knet line %d"
                      % (self.gen.cexpr(f["cond"]), f["line"]))
                    w("    " + rows)
                    w("  }")
            w("  return m;")
            w("}")
        self.pnames = pn
        self.meta = dict(
            network=net.name, key=self.key, species=list(self.species),
            mass_g=mass_g, charge=charge, params=pn,
            defaults=[None if d is None else d for d in dflt],
            required_by={s: gen.param_required_by.get(s, "") for s in pn
                         if s in req},
            nrea=nr, options=self.cfg,
            elements=self.meta_elements[0],
            species_elements=self.meta_elements[1])
        w("")

    def emit_physics(self):
        self.w('#include "../csrc/kb_physics.h"')
        self.w('#include "../csrc/kb_conserve.h"')
        self.w('#include "../csrc/kb_jacdk.h"')
        self.w("")

    def emit_vars(self):
        net = self.net
        order = getattr(net, "var_order", None) or list(net.vars)
        for name in order:
            ast = net.vars[name]
            self.w("KB_HD inline double v_%s(double Tgas, const double* n, "
                   "const Params& p) {" % name)
            self.w("  (void)Tgas; (void)n; (void)p;")
            self.w("  return %s;" % self.cx(ast, "Tgas"))
            self.w("}")
        self.w("")

    def _rate_body(self, rx, tv):
        i = rx["id"] - 1
        return ["k[%d] = %s;  // %s" % (i, self.cx(rx["rate"]["ast"], tv),
                                         rx["eq"])]

    def hoist(self, rxs, tvar, indent):
        """the vars the given rates reference, as locals of this scope"""
        names = sorted({nd["s"] for rx in rxs
                        for nd in self.gen.deep_walk(rx["rate"]["ast"])
                        if nd.get("kind") == "var"})
        self.hoisted = {}
        for s in names:
            self.w("%sconst double vh_%s = v_%s(%s, n, p);" % (indent, s, s, tvar))
            self.w("%s(void)vh_%s;" % (indent, s))
        self.hoisted = {s: "vh_" + s for s in names}

    def emit_grouped(self, body, select, hoist=True):
        """statements for the selected expr-rate reactions, singles first,
        then each piecewise group with the outside=asym selection (zero
        below the group's range, temperature clamped above it)"""
        w = self.w
        singles, groups = [], {}
        for rx in self.net.reactions:
            if rx["rate"]["kind"] != "expr" or not select(rx):
                continue
            if rx.get("group") is None:
                singles.append(rx)
            else:
                groups.setdefault(rx["group"], []).append(rx)
        if hoist and singles:
            self.hoist(singles, "Tgas", "  ")
        for rx in singles:
            for ln in body(rx, "Tgas"):
                w("  " + ln)
        self.hoisted = {}
        outside = self.gen.outside
        for g, pieces in sorted(groups.items()):
            pieces.sort(key=lambda r: r["trange"])
            glo, ghi = pieces[0]["trange"][0], pieces[-1]["trange"][1]
            w("  {  // group %d: %s" % (g, pieces[0]["eq"]))
            w("    double T = Tgas;")
            clamp_lo = outside == "clamp"
            zero_lo = outside in ("zero", "asym") and glo > 0.0
            clamp_hi = outside in ("clamp", "asym")
            if clamp_lo and glo > 0.0:
                w("    if (T < %s) T = %s;" % (self.num(glo), self.num(glo)))
            if clamp_hi and ghi != math.inf:
                w("    if (T > %s) T = %s;" % (self.num(ghi), self.num(ghi)))
            if hoist:
                self.hoist(pieces, "T", "    ")
            cond0 = "T >= %s && " % self.num(glo) if zero_lo else ""
            for j, rx in enumerate(pieces):
                lo, hi = rx["trange"]
                last = j == len(pieces) - 1
                cmp_hi = "<=" if (last and hi != math.inf) else "<"
                conds = []
                if j > 0 or zero_lo:
                    conds.append("T >= %s" % self.num(lo))
                if hi != math.inf and not (last and clamp_hi):
                    conds.append("T %s %s" % (cmp_hi, self.num(hi)))
                cond = " && ".join(conds) if conds else "true"
                kw = "if" if j == 0 else "else if"
                w("    %s (%s%s) {" % (kw, cond0 if j == 0 else "", cond))
                for ln in body(rx, "T"):
                    w("      " + ln)
                w("    }")
                cond0 = ""
            w("  }")
            self.hoisted = {}

    def emit_rates(self):
        gen = self.gen
        fixed = [rx for rx in self.net.reactions
                 if rx["rate"]["kind"] == "expr" and gen.rate_is_fixed(rx)]
        self.nfixed = len(fixed)
        for part, sel in (("fixed", gen.rate_is_fixed),
                          ("var", lambda rx: not gen.rate_is_fixed(rx))):
            self.w("// rate coefficients of Tgas and the parameters only"
                   if part == "fixed" else
                   "// rate coefficients that also depend on the densities")
            self.w("KB_HD inline void rates_%s(double Tgas, const double* n, "
                   "const Params& p, double* k) {" % part)
            self.w("  (void)Tgas; (void)n; (void)p; (void)k;")
            self.emit_grouped(self._rate_body, sel)
            if part == "var":
                for j, rx in enumerate(self.photo_rx):
                    self.w("  k[%d] += p.kph[%d];  // %s" % (rx["id"] - 1, j, rx["eq"]))
            self.w("}")
        # which coefficients each part writes
        fixed_ids = sorted(rx["id"] - 1 for rx in fixed)
        self.w("constexpr int NREA_FIXED = %d;" % len(fixed_ids))
        self.w("KB_HD inline bool rate_is_fixed(int r) {")
        self.w("  switch (r) {")
        for i in fixed_ids:
            self.w("    case %d:" % i)
        if fixed_ids:
            self.w("      return true;")
        self.w("    default: return false;")
        self.w("  }")
        self.w("}")
        self.w("")

    def _kin(self, rx):
        return [r["sp"] for r in rx["reactants"] if r["kinetic"]]

    def emit_rhs(self):
        w = self.w
        w("// mass-action dn/dt: per species, the flux terms in reaction "
          "order")
        w("KB_HD inline void rhs(const double* n, const double* k, double* dn) {")
        w("KB_UNROLL")
        w("  for (int i = 0; i < NSPEC; ++i) dn[i] = 0.0;")
        w("  double flux;")
        w("  (void)flux;")
        for rx in self.net.reactions:
            i = rx["id"] - 1
            fac = ["k[%d]" % i] + [self.den(s) for s in self._kin(rx)]
            w("  flux = %s;" % "*".join(fac))
            for r in rx["reactants"]:
                w("  dn[IDX_%s] -= flux;" % self.cid(r["sp"]))
            for pr in rx["products"]:
                w("  dn[IDX_%s] += flux;" % self.cid(pr["sp"]))
        w("}")
        w("")

    def emit_jac(self):
        """d dn_i / d n_j of the mass-action terms at fixed k, into
        J[i*rs + j*cs] (the species block, zeroed here)"""
        w = self.w
        w("KB_HD inline void jac_stoich(const double* n, const double* k, "
          "double* J, int rs, int cs) {")
        w("  for (int i = 0; i < NSPEC; ++i)")
        w("    for (int j = 0; j < NSPEC; ++j) J[i*rs + j*cs] = 0.0;")
        w("  double d;")
        w("  (void)d; (void)n; (void)k;")
        for rx in self.net.reactions:
            i = rx["id"] - 1
            targets = {}
            for s in self._kin(rx):
                targets[s] = targets.get(s, 0) + 1
            for tgt, mult in sorted(targets.items()):
                rest = ["k[%d]" % i]
                for s, c in sorted(targets.items()):
                    rest += [self.den(s)] * (c - 1 if s == tgt else c)
                coef = ("%d.0*" % mult) if mult > 1 else ""
                w("  d = %s;" % (coef + "*".join(rest)))
                col = "IDX_%s" % self.cid(tgt)
                for r in rx["reactants"]:
                    w("  J[IDX_%s*rs + %s*cs] -= d;" % (self.cid(r["sp"]), col))
                for pr in rx["products"]:
                    w("  J[IDX_%s*rs + %s*cs] += d;" % (self.cid(pr["sp"]), col))
        w("}")
        w("")

    def emit_jac_dk(self):
        """the analytic Jacobian's rate-derivative part: d k_r / d n_j prod n
        into J and d k_r / d aggregate prod n into U (J += U W^T after), in
        the reference's jacobian_split form (kromex/codegen.py:8462-8560):
        the derivative expressions and J / U updates are the reference
        generator's own rendering (jac_dk_lines), gated by the same
        piecewise selection as the rates; a rate that calls a fitted
        function is re-evaluated (rate_<r>) for difference quotients"""
        w, gen = self.w, self.gen
        for rx in self.net.reactions:
            if rx["rate"]["kind"] != "expr" or not gen.has_extern(rx["rate"]["ast"]):
                continue
            # the rate function the difference quotients call: Tgas the
            # (group-clamped) rate temperature, Tg_ the gas temperature
            w("// %s" % rx["eq"])
            w("KB_HD inline double rate_%d(double Tgas, const double* n, "
              "const Params& p, double Tg_) {" % (rx["id"] - 1))
            w("  (void)Tgas; (void)n; (void)p; (void)Tg_;")
            gen._hoisted = {}
            gen._in_ratefn = True
            try:
                w("  return %s;" % gen.cexpr(rx["rate"]["ast"])
                  .replace("constants::", "kbc::"))
            finally:
                gen._in_ratefn = False
            w("}")
        w("// the rate-derivative part of the analytic Jacobian (J[i*jrs_ + "
          "j*cs], added to;")
        w("// U[NSPEC][NAGG] written), gated and clamped like the rates")
        w("KB_HD inline void jac_dk(double Tgas, const double* n, "
          "const Params& p, const double* k, double* J, double* U, "
          "long jrs_, long jcs_) {")
        w("  (void)Tgas; (void)n; (void)p; (void)k; (void)J; (void)jrs_; "
          "(void)jcs_;")
        w("  for (int i = 0; i < NSPEC * NAGG; ++i) U[i] = 0.0;")
        w("  double d;")
        w("  (void)d;")
        def body(rx, tv):
            gen._hoisted = {}
            gen._in_ratefn = False
            return [ln.replace("constants::", "kbc::")
                    for ln in gen.jac_dk_lines(rx, tv)]
        self.emit_grouped(body, lambda rx: True, hoist=False)
        w("}")
        w("")

    # -- thermal -----------------------------------------------------------

    def _recomb_reactions(self):
        """the electron recombinations X^q+ + e- -> X^(q-1)+ of atomic ions
        the ATOMIC recombination cooling counts (reference:
        kromex/codegen.py:6857-6888)"""
        net, out = self.net, []
        for rx in net.reactions:
            if rx["rate"]["kind"] != "expr":
                continue
            R, P = rx["reactants"], rx["products"]
            if len(R) != 2 or len(P) != 1:
                continue
            ions = [r["sp"] for r in R if r["sp"] != "e-"]
            if len(ions) != 1 or len(R) - len(ions) != 1:
                continue
            ion, prod = ions[0], P[0]["sp"]
            si, sp = net.species[ion], net.species[prod]
            if si["opaque"] or sp["opaque"] or si["phase"] != "gas" \
                    or sp["phase"] != "gas" or self.gen._natoms(ion) != 1:
                continue
            if si["composition"] != sp["composition"] \
                    or sp["charge"] != si["charge"] - 1 or si["charge"] < 1:
                continue
            if any(nd.get("kind") in ("extern", "table")
                   and "dust" in str(nd.get("f", "")).lower()
                   or nd.get("s") == "Tdust"
                   for nd in self.gen.deep_walk(rx["rate"]["ast"])):
                continue
            out.append(rx)
        return out

    def _chem_terms(self):
        """the H2 chemistry ledger (thermal CHEM): (heating, cooling)
        terms as (energy in eV, reaction, critical-density factor)"""
        chem = []
        for rx in self.net.reactions:
            R = sorted(r["sp"] for r in rx["reactants"])
            P = sorted(p0["sp"] for p0 in rx["products"])
            for rr, pp, q, ff in CHEM_LEDGER:
                if R == rr and P == pp:
                    chem.append((q, rx, ff))
                    break
        return ([x for x in chem if not x[0].startswith("-")],
                [x for x in chem if x[0].startswith("-")])

    def emit_thermal(self):
        w = self.w
        th = self.gen.thermal
        net = self.net
        heat_terms, diss_terms = self._chem_terms()
        if th.get("cool_chem"):
            w("KB_HD inline double cooling_chem(const double* n, const double* k) {")
            w("  double c = 0.0;")
            for q, rx, _ in diss_terms:
                prod = "*".join(self.den(r["sp"]) for r in rx["reactants"])
                w("  c += k[%d] * %s * %s;" % (rx["id"] - 1, q[1:], prod))
            if diss_terms:
                w("  c *= kbc::eV_to_erg;")
            w("  return c;")
            w("}")
        if th.get("heat_chem"):
            w("KB_HD inline double heating_chem(double Tgas, const double* n, "
              "const double* k) {")
            w("  double h = 0.0;")
            if heat_terms:
                w("  const double ev2erg = kbc::eV_to_erg;")
                w("  const double dd = Hnuclei_(n);")
                w("  const double ncr = 1.0e6 / std::sqrt(Tgas)")
                w("      / (1.6 * std::exp(-std::pow(4.0e2 / Tgas, 2.0)) "
                  "* n[IDX_H] / dd")
                w("         + 1.4 * std::exp(-1.2e4 / (Tgas + 1.2e3)) "
                  "* n[IDX_H2] / dd);")
                w("  const double ffac = 1.0 / (1.0 + ncr / dd);")
                for q, rx, ff in heat_terms:
                    prod = "*".join(self.den(r["sp"]) for r in rx["reactants"])
                    qexpr = "%s*ffac" % q if ff else q
                    w("  h += k[%d] * (%s) * %s;" % (rx["id"] - 1, qexpr, prod))
                w("  h *= ev2erg;")
            w("  return h;")
            w("}")
        if th.get("cool_atomic"):
            rxs = self._recomb_reactions()
            idx = {rx["id"]: j for j, rx in enumerate(rxs)}
            nr = max(len(rxs), 1)
            w("// recombination rates of the ATOMIC cooling and T dk/dT of the")
            w("// piece active at T (central difference, relative step 1e-4;")
            w("// 0 where the rate's temperature is clamped)")
            w("KB_HD inline void recomb_rates_(double Tgas, const double* n, "
              "const Params& p, double* kr, double* tdk) {")
            w("  (void)n; (void)p;")
            w("  const double h = 1e-4;")
            w("  for (int j = 0; j < %d; ++j) kr[j] = tdk[j] = 0.0;" % len(rxs))

            def body(rx, tv):
                j = idx[rx["id"]]
                e = lambda t: self.cx(rx["rate"]["ast"], t)
                out = ["kr[%d] = %s;" % (j, e(tv))]
                if tv == "Tgas":
                    out.append("{ const double Tp_ = Tgas * (1.0 + h), "
                               "Tm_ = Tgas * (1.0 - h);")
                else:
                    out.append("if (%s == Tgas) { const double Tp_ = %s * "
                               "(1.0 + h), Tm_ = %s * (1.0 - h);"
                               % (tv, tv, tv))
                out.append("  tdk[%d] = ((%s) - (%s)) / (2.0 * h); }"
                           % (j, e("Tp_"), e("Tm_")))
                return out
            self.emit_grouped(body, lambda rx: rx["id"] in idx, hoist=False)
            w("}")
            w("KB_HD inline double cooling_recomb_(double Tgas, const double* n, "
              "const Params& p) {")
            w("  const double T = std::fmin(std::fmax(Tgas, p.Tcmb), 1e9);")
            w("  double k0[%d], tdk[%d];" % (nr, nr))
            w("  recomb_rates_(T, n, p, k0, tdk);")
            w("  double c = 0.0;")
            for j, rx in enumerate(rxs):
                ion = [r["sp"] for r in rx["reactants"] if r["sp"] != "e-"][0]
                w("  c += n[IDX_E] * %s * std::fmax(0.0, 1.5 * k0[%d] + tdk[%d]);"
                  % (self.den(ion), j, j))
            w("  return kbc::boltzmann_erg * T * c;")
            w("}")
            # the same from rates evaluated before (thermal_pre)
            w("KB_HD inline double cooling_recomb_with_(const double* k0, "
              "const double* tdk, double Tgas, const double* n, const Params& p) {")
            w("  const double T = std::fmin(std::fmax(Tgas, p.Tcmb), 1e9);")
            w("  double c = 0.0;")
            for j, rx in enumerate(rxs):
                ion = [r["sp"] for r in rx["reactants"] if r["sp"] != "e-"][0]
                w("  c += n[IDX_E] * %s * std::fmax(0.0, 1.5 * k0[%d] + tdk[%d]);"
                  % (self.den(ion), j, j))
            w("  return kbc::boltzmann_erg * T * c;")
            w("}")
            self.n_recomb = nr
        if th.get("cool_H2"):
            mode = self.gen.h2_opacity
            w("KB_HD inline double h2_opacity_(const double* n) {")
            w("  (void)n;")
            if mode == "RIPAMONTI":
                w("  return std::fmin(1.0, std::pow(std::fmax(1.25e-10 * "
                  "ntot_(n), 1e-40), -0.45));")
            elif not mode:
                w("  return 1.0;")
            else:
                raise NotImplementedError("h2_opacity %s" % mode)
            w("}")
        self.emit_gamma()
        # dT/dt
        w("// dTgas/dt at the thermal temperature T (capped to [2.73, 1e9] K by")
        w("// the caller) with the rates k of the rate temperature")
        w("KB_HD inline double thermal_dTdt(double T, const double* n, "
          "const double* k, const Params& p) {")
        w("  (void)k; (void)p;")
        w("  double heat = 0.0, cool = 0.0;")
        heat_order = [("heat_CR", None), ("heat_chem", "heating_chem(T, n, k)"),
                      ("heat_dH", None),
                      ("heat_compress", "ntot_(n) * kbc::boltzmann_erg * T / p.tff")]
        supported = {"heat_chem", "heat_compress"}
        for f, expr in heat_order:
            if th.get(f):
                if f not in supported:
                    raise NotImplementedError(f)
                w("  heat += %s;" % expr)
        for f in ("heat_visc", "heat_photoDust", "heat_netPhotoDust",
                  "heat_photoAv", "heat_photo", "heat_ZCIE", "heat_nuclear"):
            if th.get(f):
                raise NotImplementedError(f)
        cool_order = [
            ("cool_atomic", "cooling_Atomic(T, n) + cooling_recomb_(T, n, p)"),
            ("cool_H2", "cooling_H2(T, n) * h2_opacity_(n)"),
            ("cool_chem", "cooling_chem(n, k)"),
            ("cool_cont", "cooling_Continuum(T, n)"),
        ]
        for f in ("cool_HD", "cool_mol", "cool_Z", "cool_ZCIE", "cool_Zext",
                  "cooling_floor", "cool_compton", "cool_CIE", "cool_expansion",
                  "cool_ff", "cool_dH", "cool_dust", "cool_dustTab",
                  "cool_dust_bins"):
            if th.get(f):
                raise NotImplementedError(f)
        for f, expr in cool_order:
            if th.get(f):
                w("  cool += %s;" % expr)
        w("  return (gamma_index(T, n, p) - 1.0) * (heat - cool)")
        w("      / (kbc::boltzmann_erg * ntot_(n));")
        w("}")
        # the temperature-only parts of the cooling at T, and dTgas/dt from
        # them: thermal_dTdt_with(thermal_pre(T), T, n, k, p) ==
        # thermal_dTdt(T, n, k, p) bit for bit (a row of density
        # derivatives at one T evaluates them once)
        atomic, h2 = th.get("cool_atomic"), th.get("cool_H2")
        w("// the cooling's temperature-only parts at one T (a row of density")
        w("// derivatives at that T evaluates them once): thermal_dTdt_with of")
        w("// thermal_pre(T) equals thermal_dTdt bit for bit")
        w("struct ThermalPre {")
        if atomic:
            w("  CoolAtomicC atomic;")
            w("  double k0[%d], tdk[%d];" % (self.n_recomb, self.n_recomb))
        if h2:
            w("  CoolH2C h2;")
        w("  int unused_;")
        w("};")
        w("KB_HD inline void thermal_pre(double T, const double* n, "
          "const Params& p, ThermalPre& q) {")
        w("  (void)T; (void)n; (void)p; (void)q;")
        if atomic:
            w("  q.atomic = cooling_Atomic_coef(T);")
            w("  recomb_rates_(std::fmin(std::fmax(T, p.Tcmb), 1e9), n, p, "
              "q.k0, q.tdk);")
        if h2:
            w("  q.h2 = cooling_H2_coef(T);")
        w("}")
        w("KB_HD inline double thermal_dTdt_with(const ThermalPre& q, double T, "
          "const double* n, const double* k, const Params& p) {")
        w("  (void)q; (void)k; (void)p;")
        w("  double heat = 0.0, cool = 0.0;")
        for f, expr in heat_order:
            if th.get(f):
                w("  heat += %s;" % expr)
        with_ = {
            "cool_atomic": "cooling_Atomic_with(q.atomic, n) + "
                           "cooling_recomb_with_(q.k0, q.tdk, T, n, p)",
            "cool_H2": "cooling_H2_with(q.h2, n) * h2_opacity_(n)",
        }
        for f, expr in cool_order:
            if th.get(f):
                w("  cool += %s;" % with_.get(f, expr))
        w("  return (gamma_index(T, n, p) - 1.0) * (heat - cool)")
        w("      / (kbc::boltzmann_erg * ntot_(n));")
        w("}")
        w("")

    def emit_gamma(self):
        """the adiabatic index: CONST (the gamma_ad parameter) or EXACT
        (reference: kromex/codegen.py:3697-3819)"""
        w = self.w
        gen = self.gen
        mode = gen.gamma
        if mode == "CONST":
            w("KB_HD inline double gamma_index(double Tgas, const double* n, "
              "const Params& p) {")
            w("  (void)Tgas; (void)n;")
            w("  return p.gamma_ad;")
            w("}")
            return
        if mode != "EXACT":
            raise NotImplementedError("gamma %s" % mode)
        cg = self.cg
        sp_sorted = self.species
        mono = [s for s in sp_sorted if gen._natoms(s) == 1]
        dis = []
        for s in sp_sorted:
            if gen._natoms(s) != 2:
                continue
            ve, be = cg.GAMMA_VIB_K.get(s), cg.GAMMA_ROT_K.get(s)
            if ve is None and be is None:
                continue
            dis.append((s, ve, be))
        ves = [ve for _, ve, _ in dis if ve is not None]
        if any(be is not None for s, _, be in dis if s != "H2"):
            w("KB_HD inline double gamma_rot_(double Tin, double brot) {")
            w("  const double ib = brot / std::fmax(Tin, 10.0);")
            w("  double z = 0.0, e1 = 0.0, e2 = 0.0;")
            w("KB_UNROLL")
            w("  for (int j = 0; j <= 10; ++j) {")
            w("    const double E = j * (j + 1.0) * ib;")
            w("    const double g = (2.0 * j + 1.0) * std::exp(-E);")
            w("    z += g; e1 += g * E; e2 += g * E * E;")
            w("  }")
            w("  const double m = e1 / z;")
            w("  return e2 / z - m * m;")
            w("}")
        if any(s == "H2" and be is not None for s, _, be in dis):
            w("KB_HD inline double gamma_rotop_(double Tin, double a) {")
            w("  const double ib = 85.4 / std::fmax(Tin, 10.0);")
            w("  double zp = 0.0, p1 = 0.0, p2 = 0.0, zo = 0.0, o1 = 0.0, "
              "o2 = 0.0;")
            w("KB_UNROLL")
            w("  for (int j = 0; j <= 10; j += 2) {")
            w("    const int j1 = j + 1;")
            w("    const double Ep = j * (j + 1.0) * ib;")
            w("    const double Eo = j1 * (j1 + 1.0) * ib;")
            w("    const double gp = (2.0 * j + 1.0) * std::exp(-Ep);")
            w("    const double go = 3.0 * (2.0 * j1 + 1.0) * std::exp(-Eo);")
            w("    zp += gp; p1 += gp * Ep; p2 += gp * Ep * Ep;")
            w("    zo += go; o1 += go * Eo; o2 += go * Eo * Eo;")
            w("  }")
            w("  const double b = 1.0 - a;")
            w("  const double mp = p1 / zp, mo = o1 / zo;")
            w("  return b * (p2 / zp - mp * mp) + a * (o2 / zo - mo * mo);")
            w("}")
        w("KB_HD inline double gamma_index(double Tgas, const double* n, "
          "const Params& p) {")
        w("  (void)Tgas; (void)n; (void)p;")
        if ves:
            w("  const double iTv = 1.0 / std::fmax(Tgas, %s);"
              % self.num(min(ves) * 1e-2))
        terms = []
        for s, ve, be in dis:
            cs = self.cid(s)
            vpart = "0.0"
            if ve is not None:
                w("  const double x_%s = %s * iTv, e_%s = std::exp(x_%s);"
                  % (cs, self.num(ve), cs, cs))
                vpart = ("2.0 * x_%s * x_%s * e_%s / ((e_%s - 1.0) * "
                         "(e_%s - 1.0))" % (cs, cs, cs, cs, cs))
            rpart = "2.0"
            if be is not None:
                rpart = ("2.0 * gamma_rotop_(Tgas, p.opratio / (p.opratio + 1.0))"
                         if s == "H2"
                         else "2.0 * gamma_rot_(Tgas, %s)" % self.num(be))
            w("  const double gi_%s = 0.5 * (3.0 + %s + %s);" % (cs, rpart, vpart))
            terms.append(cs)
        w("  const double mosum = %s;"
          % (" + ".join(self.den(s) for s in mono) or "0.0"))
        w("  const double ysum = mosum%s;"
          % "".join(" + n[IDX_%s]" % c for c in terms))
        w("  const double gsum = 1.5 * mosum%s;"
          % "".join(" + n[IDX_%s] * gi_%s" % (c, c) for c in terms))
        w("  return gsum > 0.0 ? 1.0 + ysum / gsum : 5.0 / 3.0;")
        w("}")

    def emit_lnk_vjp(self):
        """the contraction of d f / d ln k with a vector mu, for the
        adjoint's per-reaction ln-multipliers: f is linear in each rate
        coefficient (the mass-action fluxes and the chemical heating and
        cooling), so d f_i / d ln k_r is reaction r's own term of f_i"""
        w = self.w
        th = self.gen.thermal
        w("// g[r] += sum_i mu_i d f_i / d ln k_r at the state n with the rates k;")
        w("// muT: mu of the Tgas row (0 without it), Tth the thermal temperature")
        w("KB_HD inline void lnk_vjp(const double* n, const double* k, double Tth, "
          "const Params& p, const double* mu, double muT, double* g) {")
        w("  (void)Tth; (void)p; (void)muT;")
        w("  double flux;")
        w("  (void)flux;")
        for rx in self.net.reactions:
            i = rx["id"] - 1
            fac = ["k[%d]" % i] + [self.den(s) for s in self._kin(rx)]
            terms = (["+ mu[IDX_%s]" % self.cid(pr["sp"]) for pr in rx["products"]]
                     + ["- mu[IDX_%s]" % self.cid(r["sp"]) for r in rx["reactants"]])
            if not terms:
                continue
            w("  flux = %s;" % "*".join(fac))
            w("  g[%d] += flux * (%s);" % (i, " ".join(terms).lstrip("+ ")))
        heat_terms, diss_terms = self._chem_terms()
        heat = th.get("heat_chem") and heat_terms
        cool = th.get("cool_chem") and diss_terms
        if heat or cool:
            w("  if (muT != 0.0) {")
            w("    const double c = muT * (gamma_index(Tth, n, p) - 1.0)"
              " / (kbc::boltzmann_erg * ntot_(n)) * kbc::eV_to_erg;")
            if cool:
                for q, rx, _ in diss_terms:
                    prod = "*".join(self.den(r["sp"]) for r in rx["reactants"])
                    w("    g[%d] -= c * k[%d] * %s * %s;"
                      % (rx["id"] - 1, rx["id"] - 1, q[1:], prod))
            if heat:
                w("    const double dd = Hnuclei_(n);")
                w("    const double ncr = 1.0e6 / std::sqrt(Tth)")
                w("        / (1.6 * std::exp(-std::pow(4.0e2 / Tth, 2.0)) "
                  "* n[IDX_H] / dd")
                w("           + 1.4 * std::exp(-1.2e4 / (Tth + 1.2e3)) "
                  "* n[IDX_H2] / dd);")
                w("    const double ffac = 1.0 / (1.0 + ncr / dd);")
                w("    (void)ffac;")
                for q, rx, ff in heat_terms:
                    prod = "*".join(self.den(r["sp"]) for r in rx["reactants"])
                    qexpr = "%s*ffac" % q if ff else q
                    w("    g[%d] += c * k[%d] * (%s) * %s;"
                      % (rx["id"] - 1, rx["id"] - 1, qexpr, prod))
            w("  }")
        w("}")
        w("")

    # -- grain-surface chemistry ------------------------------------------

    def emit_surface(self):
        """the surface processes the rates call (adsorption, thermal and
        cosmic-ray desorption, Langmuir-Hinshelwood two-body reactions),
        restated from the generator's resolved surface data: binding
        energies (bare / water ice), barriers, branching and reactive
        desorption per reaction. One grain population (the network's
        surface_grains single(n, a2)); the dust temperature the rates see is
        the Tdust parameter (no dust tables)."""
        gen, net, w = self.gen, self.net, self.w
        surfs = getattr(gen, "_surf", None) or []
        if not surfs:
            return
        sg = net.surface_grains
        if sg is None or sg.get("kind") != "single" or gen.surface_bins:
            raise NotImplementedError("surface chemistry on binned dust")
        sp_sorted = self.species
        base = {x: gen.surf_base(x) for x in sp_sorted}
        eb = gen._surf_eb
        ice = [x for x in sp_sorted if net.species[x]["phase"] != "gas"
               and base[x] == "H2O" and net.species[x]["label"] != "c"]
        self.ice_idx = self.idx[ice[0]] if ice else -1
        legacy_nu = gen.surface_nu == "LEGACY"
        w("// ---- grain-surface chemistry (binding energies %s, vibration"
          % gen.binding_energies)
        w("// frequency %s, E_diff = %s E_bind, competition %s, tunnelling %s)"
          % ("1e12 s^-1" if legacy_nu else "sqrt(2 n_s E_b / (pi^2 m))",
             self.num(gen.FDIFF[gen.binding_energies]),
             "on" if gen.surface_competition else "off",
             "on" if gen.surface_tunnelling else "off"))
        w("namespace surf {")
        w("constexpr double SITE_AREA = %s;  // [cm^2]" % self.num(gen.SURF_APP2))
        w("constexpr double FDIFF = %s;" % self.num(gen.FDIFF[gen.binding_energies]))
        w("// surface sites per volume: 4 pi n_grain a^2 / site area")
        w("KB_HD inline double sites(const Params& p) {")
        w("  return 4.0 * kbc::pi * (%s) * (%s) / SITE_AREA;"
          % (self.cx(sg["n"], "Tgas"), self.cx(sg["a2"], "Tgas")))
        w("}")
        w("// water-ice coverage in monolayers, within [0, 1]")
        w("KB_HD inline double ice_cover(const double* n, double S) {")
        if ice:
            w("  if (!(S > 0.0)) return 0.0;")
            w("  return fmin(fmax(%s / S, 0.0), 1.0);" % self.den(ice[0]))
        else:
            w("  (void)n; (void)S;")
            w("  return 0.0;")
        w("}")
        w("KB_HD inline double nu(double mass_g, double Eb) {")
        if legacy_nu:
            w("  (void)mass_g; (void)Eb;")
            w("  return 1e12;")
        else:
            w("  return sqrt(2.0 / SITE_AREA * Eb * kbc::boltzmann_erg "
              "/ (kbc::pi * kbc::pi * mass_g));")
        w("}")
        # binding energies per species (bare, ice), a switch for device code
        w("KB_HD inline void binding(int sp, double& bare, double& icy) {")
        w("  switch (sp) {")
        for i, x in enumerate(sp_sorted):
            e = eb.get(base[x])
            if e is not None and (e[0] != 0.0 or e[1] != 0.0):
                w("  case %d: bare = %s; icy = %s; return;"
                  % (i, self.num(e[0]), self.num(e[1])))
        w("  default: bare = 0.0; icy = 0.0; return;")
        w("  }")
        w("}")
        w("}  // namespace surf")
        kinds = {x["kind"] for x in surfs}
        vth = self.num(math.sqrt(8.0 * kbc_boltzmann_erg / math.pi))
        if "ads_s" in kinds:
            w("// adsorption, without the sticking factor [1/s]: the thermal")
            w("// speed times the grains' cross section pi n a^2 = S site/4")
            w("KB_HD inline double surf_adsorption_ns(int sp, double binf, "
              "double Tgas, const double* n, const Params& p) {")
            w("  (void)binf; (void)n;")
            w("  return %s * sqrt(Tgas / species_mass_g(sp)) * surf::sites(p) "
              "* surf::SITE_AREA * 0.25;" % vth)
            w("}")
        if "des" in kinds:
            cr = gen.cr_desorption
            w("// thermal desorption nu exp(-E/Td) over the bare and the icy")
            w("// fractions of the surface%s"
              % (", plus cosmic-ray spot heating (Hasegawa & Herbst 1993:"
                 if cr else ""))
            if cr:
                w("// the 70 K rate times 3.16e-19 %s / 1.3e-17)" % cr)
            w("KB_HD inline double surf_desorption(int sp, double binf, "
              "double Tgas, const double* n, const Params& p) {")
            w("  (void)binf; (void)Tgas;")
            w("  const double fi = surf::ice_cover(n, surf::sites(p));")
            w("  double Eb, Ei;")
            w("  surf::binding(sp, Eb, Ei);")
            w("  const double m = species_mass_g(sp);")
            w("  const double vb = surf::nu(m, Eb), vi = surf::nu(m, Ei);")
            w("  const double Td = p.Tdust;")
            w("  double k = (1.0 - fi) * vb * exp(-Eb / Td) + fi * vi * exp(-Ei / Td);")
            if cr:
                w("  k += 3.16e-19 * p.%s / 1.3e-17 * ((1.0 - fi) * vb * "
                  "exp(-Eb / 70.0) + fi * vi * exp(-Ei / 70.0));" % cr)
            w("  return k;")
            w("}")
        hbar = gen.HBAR
        for q, x in enumerate(surfs):
            if x["kind"] != "2body":
                continue
            A, B = x["A"], x["B"]
            def spc(b):
                return b if b in net.species else next(
                    y for y in sp_sorted if base[y] == b)
            sA, sB = spc(A), spc(B)
            rx = x["rx"]
            same = rx["reactants"][0]["sp"] == rx["reactants"][1]["sp"]
            eA = eb.get(base[sA], (0.0, 0.0))
            eB = eb.get(base[sB], (0.0, 0.0))
            if "Ea" in x:
                Ea = x["Ea"]
                if Ea <= 0:
                    prob = "1.0"
                elif gen.surface_tunnelling:
                    mA = net.species[sA]["mass_amu"] * kbc_amu
                    mB = net.species[sB]["mass_amu"] * kbc_amu
                    mu = mA * mB / (mA + mB)
                    tun = math.exp(-2.0 * gen.SURF_TUNNEL_A / hbar
                                   * math.sqrt(2.0 * mu * Ea * kbc_boltzmann_erg))
                    prob = "fmax(exp(-%s / Td), %s)" % (self.num(Ea), self.num(tun))
                else:
                    prob = "exp(-%s / Td)" % self.num(Ea)
            else:
                prob = self.num(x["prob"])
            cdb, cdi = x["cd"]
            w("// %s: Langmuir-Hinshelwood%s; mode 0 the whole rate, 1 the"
              % (rx["eq"], ", identical reactants (1/2)" if same else ""))
            w("// surface branch (1 - f), 2 the desorbing branch (f), f the")
            w("// reactive desorption fraction")
            w("KB_HD inline double surf_2body_%d(double mode, double binf, "
              "double Tgas, const double* n, const Params& p) {" % q)
            w("  (void)binf; (void)Tgas;")
            w("  const double S = surf::sites(p);")
            w("  if (!(S > 0.0)) return 0.0;")
            w("  const double fi = surf::ice_cover(n, S), fb = 1.0 - fi;")
            w("  const double Td = p.Tdust;")
            w("  const double mA = species_mass_g(IDX_%s), mB = species_mass_g(IDX_%s);"
              % (self.cid(sA), self.cid(sB)))
            w("  (void)mA; (void)mB;")
            w("  const double prob = %s;" % prob)
            w("  auto k1 = [&](double EA, double EB) {")
            w("    const double nA = surf::nu(mA, EA), nB = surf::nu(mB, EB);")
            w("    const double hA = nA * exp(-surf::FDIFF * EA / Td);")
            w("    const double hB = nB * exp(-surf::FDIFF * EB / Td);")
            if gen.surface_competition:
                w("    const double Pr = fmax(nA, nB) * prob;")
                w("    const double den = Pr + hA + hB + nA * exp(-EA / Td) "
                  "+ nB * exp(-EB / Td);")
                w("    const double kap = den > 0.0 ? Pr / den : 0.0;")
            else:
                w("    const double kap = prob;")
            w("    return kap * (hA + hB);")
            w("  };")
            w("  double k = %s * (fb * k1(%s, %s) + fi * k1(%s, %s)) / S;"
              % (self.num(x["branch"] * (0.5 if same else 1.0)),
                 self.num(eA[0]), self.num(eB[0]), self.num(eA[1]), self.num(eB[1])))
            w("  const double f = fb * %s + fi * %s;" % (self.num(cdb), self.num(cdi)))
            w("  if (mode == 1.0) k *= 1.0 - f;")
            w("  else if (mode == 2.0) k *= f;")
            w("  return k;")
            w("}")
        w("")

    # -- the sparse path of large networks ---------------------------------

    NPART = 32  # a warp's lanes: each evaluates one part

    def _rate_units(self, select):
        """the selected expr reactions as units: singles, and whole
        piecewise groups"""
        units, groups = [], {}
        for rx in self.net.reactions:
            if rx["rate"]["kind"] != "expr" or not select(rx):
                continue
            if rx.get("group") is None:
                units.append([rx])
            else:
                if rx["group"] not in groups:
                    groups[rx["group"]] = []
                    units.append(groups[rx["group"]])
                groups[rx["group"]].append(rx)
        return units

    RPART = 256  # rate parts of a large network: one per thread of a cell's block

    def _var_closure(self, names):
        """the vars `names` and every var they reference, in the order the
        vars are defined (dependencies first)"""
        net = self.net
        need, todo = set(), list(names)
        while todo:
            v = todo.pop()
            if v in need:
                continue
            need.add(v)
            for nd in self.gen.deep_walk(net.vars[v]):
                if nd.get("kind") == "var":
                    todo.append(nd["s"])
        order = getattr(net, "var_order", None) or list(net.vars)
        return [v for v in order if v in need]

    def _hoist_inline(self, rxs, tvar, indent):
        """hoist() for the rate parts: the vars as expressions of locals,
        with the H-nuclei density the parameter hnuc (one block reduction per
        evaluation instead of a species sum in every part)"""
        names = sorted({nd["s"] for rx in rxs
                        for nd in self.gen.deep_walk(rx["rate"]["ast"])
                        if nd.get("kind") == "var"})
        self.hoisted = {}
        for v in self._var_closure(names):
            e = self.cx(self.net.vars[v], tvar).replace("Hnuclei_(n)", "hnuc")
            self.w("%sconst double vh_%s = %s;" % (indent, v, e))
            self.w("%s(void)vh_%s;" % (indent, v))
            self.hoisted[v] = "vh_" + v

    def emit_rate_parts(self):
        """rates_fixed_part / rates_var_part: the rate coefficients split
        into RPART parts (thread `part` of a cell's block computes its
        part); hnuc = Hnuclei_(n) of the same n"""
        gen = self.gen
        self.w("constexpr int RPART = %d;" % self.RPART)
        hoist0 = self.hoist
        self.hoist = self._hoist_inline
        for name, sel in (("fixed", gen.rate_is_fixed),
                          ("var", lambda rx: not gen.rate_is_fixed(rx))):
            units = self._rate_units(sel)
            part_of = {}
            for u, unit in enumerate(units):
                for rx in unit:
                    part_of[rx["id"]] = u % self.RPART
            self.w("KB_HD inline void rates_%s_part(int part, double Tgas, "
                   "const double* n, const Params& p, double hnuc, double* k) {"
                   % name)
            self.w("  (void)Tgas; (void)n; (void)p; (void)hnuc; (void)k;")
            self.w("  switch (part) {")
            for j in range(self.RPART):
                self.w("  case %d: {" % j)
                first = len(self.lines)
                self.emit_grouped(self._rate_body,
                                  lambda rx, j=j: sel(rx) and part_of.get(rx["id"]) == j)
                for q in range(first, len(self.lines)):
                    self.lines[q] = self.lines[q].replace("Hnuclei_(n)", "hnuc")
                self.w("  } break;")
            self.w("  default: break;")
            self.w("  }")
            self.w("}")
        self.hoist = hoist0
        # the density-dependent rates, and how they depend on the state:
        # through the water-ice coverage fi of the surface functions (affine
        # in fi) and the H-nuclei density (linear), nothing else -- then
        # with Tgas and Tdust fixed a solve needs each of them at three
        # points only (fi = 0, fi = 1, hnuc = 1; a test checks the form
        # against the direct evaluation)
        var_rx = [rx for rx in self.net.reactions
                  if rx["rate"]["kind"] == "expr" and not gen.rate_is_fixed(rx)]
        var = sorted(rx["id"] - 1 for rx in var_rx)
        direct = any(nd.get("kind") == "density" for rx in var_rx
                     for nd in gen.deep_walk(rx["rate"]["ast"]))
        self.w("constexpr int BK_NVAR = %d;" % len(var))
        self.w("constexpr int BK_ICE = %d;  // the ice species (-1: none)"
               % getattr(self, "ice_idx", -1))
        self.w("constexpr int BK_VAR_AFFINE = %d;" % (0 if direct else 1))
        self._table("bk_var", var or [0])
        ice = getattr(self, "ice_idx", -1)
        self.w("// the ice coverage of state n, and n with coverage 0 or 1")
        self.w("KB_HD inline double bk_ice_cover(const double* n, const Params& p) {")
        if ice >= 0:
            self.w("  return surf::ice_cover(n, surf::sites(p));")
        else:
            self.w("  (void)n; (void)p;")
            self.w("  return 0.0;")
        self.w("}")
        self.w("KB_HD inline void bk_set_ice(double* n, const Params& p, int full) {")
        if ice >= 0:
            self.w("  n[%d] = full ? surf::sites(p) : 0.0;" % ice)
        else:
            self.w("  (void)n; (void)p; (void)full;")
        self.w("}")
        self.w("")

    def _sparse_pattern(self):
        """the Newton matrix I - gamma J over the species: J_ij != 0 where
        species i takes part in a reaction with kinetic reactant j; plus the
        diagonal"""
        idx = self.idx
        pat = set((i, i) for i in range(len(self.species)))
        for rx in self.net.reactions:
            kin = set(idx[s] for s in self._kin(rx))
            aff = set(idx[r["sp"]] for r in rx["reactants"]) | \
                set(idx[p0["sp"]] for p0 in rx["products"])
            for i in aff:
                for j in kin:
                    pat.add((i, j))
        return pat

    @staticmethod
    def _min_degree(n, pat):
        """a minimum-degree elimination order of the symmetrised pattern
        (each elimination joins its neighbours into a clique: the fill)"""
        import heapq
        adj = [set() for _ in range(n)]
        for i, j in pat:
            if i != j:
                adj[i].add(j)
                adj[j].add(i)
        heap = [(len(adj[v]), v) for v in range(n)]
        heapq.heapify(heap)
        alive = set(range(n))
        order = []
        while heap:
            d, v = heapq.heappop(heap)
            if v not in alive or d != len(adj[v]):
                continue
            order.append(v)
            alive.discard(v)
            nb = adj[v]
            for u in nb:
                adj[u].discard(v)
                adj[u] |= nb - {u}
                heapq.heappush(heap, (len(adj[u]), u))
            adj[v] = set()
        return order

    @staticmethod
    def _symbolic_lu(n, rows):
        """the fill of a row-oriented (IKJ) LU without pivoting: row i gains
        the upper part of every row k < i it eliminates, in increasing k"""
        import heapq
        upper = [None] * n
        for i in range(n):
            r = rows[i]
            ks = [k for k in r if k < i]
            heapq.heapify(ks)
            seen = set(ks)
            while ks:
                k = heapq.heappop(ks)
                for j in upper[k]:
                    if j not in r:
                        r.add(j)
                        if j < i and j not in seen:
                            heapq.heappush(ks, j)
                            seen.add(j)
            upper[i] = sorted(j for j in r if j > i)
        return rows

    def _table(self, name, vals):
        body = ",".join(str(v) for v in vals)
        self.w("#define KB_T_%s %s" % (name, body))
        self.w("inline const int %s[%d] = {KB_T_%s};" % (name, len(vals), name))
        self.w("#ifdef __CUDACC__")
        self.w("__device__ const int d_%s[%d] = {KB_T_%s};" % (name, len(vals), name))
        self.w("#endif")
        self.w("#undef KB_T_%s" % name)

    def emit_sparse(self):
        """the static-pivot sparse LU structure (fixed at generation) and
        the gather forms of the flux, rhs and Jacobian, split into parts"""
        w = self.w
        n = len(self.species)
        idx = self.idx
        pat = self._sparse_pattern()
        order = self._min_degree(n, pat)
        new = {v: k for k, v in enumerate(order)}
        rows = [set() for _ in range(n)]
        for i, j in pat:
            rows[new[i]].add(new[j])
        rows = self._symbolic_lu(n, rows)
        rp, ci, di = [0], [], []
        pos = {}
        for i in range(n):
            cols = sorted(rows[i])
            for j in cols:
                pos[(i, j)] = len(ci)
                ci.append(j)
            di.append(pos[(i, i)])
            rp.append(len(ci))
        # the Jacobian's entries (original indices), sorted by their row
        ent = sorted((i, j) for i, j in pat if True)
        eidx = {e: k for k, e in enumerate(ent)}
        jpos = [pos[(new[i], new[j])] for i, j in ent]
        self.meta["nnz_lu"] = len(ci)
        self.meta["nnz_j"] = len(ent)
        w("// ---- the sparse path: static-pivot LU of I - gamma J ----")
        w("// rows / columns in the elimination order sp_perm (a minimum-degree")
        w("// order of the symmetrised pattern); the pattern includes the fill")
        w("#define KB_LARGE_NETWORK 1")
        w("constexpr int NNZ_LU = %d;" % len(ci))
        w("constexpr int NNZ_J = %d;" % len(ent))
        w("constexpr int NPART = %d;" % self.NPART)
        self._table("sp_rp", rp)
        self._table("sp_ci", ci)
        self._table("sp_di", di)
        self._table("sp_perm", order)
        self._table("sp_iperm", [new[v] for v in range(n)])
        self._table("sp_jpos", jpos)
        self._emit_block_tables(n, rp, ci, di, pos, jpos)
        w("")
        P = self.NPART
        # fluxes: fl[r] = k[r] * (kinetic reactants)
        w("KB_HD inline void flux_part(int part, const double* n, "
          "const double* k, double* fl) {")
        w("  (void)n; (void)k; (void)fl;")
        w("  switch (part) {")
        for j in range(P):
            w("  case %d:" % j)
            for rx in self.net.reactions[j::P]:
                i = rx["id"] - 1
                fac = ["k[%d]" % i] + [self.den(s0) for s0 in self._kin(rx)]
                w("    fl[%d] = %s;" % (i, "*".join(fac)))
            w("    break;")
        w("  default: break;")
        w("  }")
        w("}")
        # the rhs per species, its flux terms in reaction order (the
        # unrolled rhs's order: reactants' minus before products' plus)
        terms = [[] for _ in range(n)]
        for rx in self.net.reactions:
            i = rx["id"] - 1
            for r in rx["reactants"]:
                terms[idx[r["sp"]]].append("-= fl[%d]" % i)
            for p0 in rx["products"]:
                terms[idx[p0["sp"]]].append("+= fl[%d]" % i)
        w("KB_HD inline void rhs_gather_part(int part, const double* fl, "
          "double* f) {")
        w("  (void)fl; (void)f;")
        w("  switch (part) {")
        for j in range(P):
            w("  case %d: {" % j)
            for sidx in range(j, n, P):
                w("    { double a = 0.0;")
                for t in terms[sidx]:
                    w("      a %s;" % t)
                w("      f[%d] = a; }" % sidx)
            w("  } break;")
        w("  default: break;")
        w("  }")
        w("}")
        # the Jacobian per entry: the jac_stoich terms of entry (i, j) in
        # reaction order
        jterms = [[] for _ in ent]
        for rx in self.net.reactions:
            i = rx["id"] - 1
            targets = {}
            for s0 in self._kin(rx):
                targets[s0] = targets.get(s0, 0) + 1
            for tgt, mult in sorted(targets.items()):
                rest = ["k[%d]" % i]
                for s0, c in sorted(targets.items()):
                    rest += [self.den(s0)] * (c - 1 if s0 == tgt else c)
                coef = ("%d.0*" % mult) if mult > 1 else ""
                d = coef + "*".join(rest)
                jt = idx[tgt]
                for r in rx["reactants"]:
                    jterms[eidx[(idx[r["sp"]], jt)]].append("-= " + d)
                for p0 in rx["products"]:
                    jterms[eidx[(idx[p0["sp"]], jt)]].append("+= " + d)
        # the same three forms as tables, for evaluation with one lane per
        # reaction / species / entry (a slot n[NSPEC] = 1 pads the products)
        kinr = [[idx[s0] for s0 in self._kin(rx)] for rx in self.net.reactions]
        if max(len(x) for x in kinr) > 3:
            raise NotImplementedError("more than three kinetic reactants")
        pad = lambda x, m: x + [n] * (m - len(x))
        fx = [pad(x, 3) for x in kinr]
        self._table("fx_a", [x[0] for x in fx])
        self._table("fx_b", [x[1] for x in fx])
        self._table("fx_c", [x[2] for x in fx])
        rs_rp, rs_r, rs_s = [0], [], []
        for sidx in range(n):
            for t in terms[sidx]:
                rs_r.append(int(t.split("[")[1].split("]")[0]))
                rs_s.append(-1 if t.startswith("-") else 1)
            rs_rp.append(len(rs_r))
        self._table("rs_rp", rs_rp)
        self._table("rs_r", rs_r)
        self._table("rs_s", rs_s)
        # the same terms in chunks of at most GCHUNK (a species' chunks
        # consecutive): a thread sums a chunk, then a species its chunks in
        # order -- the hub species' hundreds of terms spread over threads
        GCHUNK = 16
        ck_t, ck_rp = [], [0]
        for sidx in range(n):
            for a in range(rs_rp[sidx], rs_rp[sidx + 1], GCHUNK):
                ck_t.append(a)
            ck_rp.append(len(ck_t))
        ck_t.append(rs_rp[n])
        w("constexpr int NCHUNK = %d;  // rhs term chunks" % (len(ck_t) - 1))
        self._table("ck_t", ck_t)
        self._table("ck_rp", ck_rp)
        jt_rp, jt_r, jt_c, jt_o0, jt_o1 = [0], [], [], [], []
        jtab = [[] for _ in ent]
        for rx in self.net.reactions:
            i = rx["id"] - 1
            targets = {}
            for s0 in self._kin(rx):
                targets[s0] = targets.get(s0, 0) + 1
            for tgt, mult in sorted(targets.items()):
                others = []
                for s0, c in sorted(targets.items()):
                    others += [idx[s0]] * (c - 1 if s0 == tgt else c)
                if len(others) > 2:
                    raise NotImplementedError("a Jacobian term of four factors")
                others = pad(others, 2)
                jt = idx[tgt]
                for r in rx["reactants"]:
                    jtab[eidx[(idx[r["sp"]], jt)]].append((i, -mult, others))
                for p0 in rx["products"]:
                    jtab[eidx[(idx[p0["sp"]], jt)]].append((i, mult, others))
        for e in range(len(ent)):
            for (i, c, o) in jtab[e]:
                jt_r.append(i)
                jt_c.append(c)
                jt_o0.append(o[0])
                jt_o1.append(o[1])
            jt_rp.append(len(jt_r))
        self._table("jt_rp", jt_rp)
        self._table("jt_r", jt_r)
        self._table("jt_c", jt_c)
        self._table("jt_o0", jt_o0)
        self._table("jt_o1", jt_o1)
        w("constexpr int NTERM_RHS = %d;" % len(rs_r))
        w("constexpr int NTERM_JAC = %d;" % len(jt_r))
        w("// Jc[e] = dF_i/dn_j of entry e = (i, j) at fixed k (sp_jpos[e]: its")
        w("// place in the LU values)")
        w("KB_HD inline void jac_gather_part(int part, const double* n, "
          "const double* k, double* Jc) {")
        w("  (void)n; (void)k; (void)Jc;")
        w("  switch (part) {")
        for j in range(P):
            w("  case %d: {" % j)
            for e in range(j, len(ent), P):
                w("    { double a = 0.0;")
                for t in jterms[e]:
                    w("      a %s;" % t)
                w("      Jc[%d] = a; }" % e)
            w("  } break;")
        w("  default: break;")
        w("  }")
        w("}")
        w("")

    BK_DMAX = 160  # the dense trailing block of a cell's LU, in shared memory

    def _emit_block_tables(self, n, rp, ci, di, pos, jpos):
        """the schedule of the block-per-cell factorization and solves: the
        first BK_M rows of the elimination order are sparse, the last BK_D
        rows and columns form a dense block S (row stride BK_LD, in shared
        memory).
          bk_frow / bk_flp   the sparse rows by forward level (a row's level
                             is one above the highest level of the rows its
                             L entries eliminate with; level 0: no L entries)
          bk_brow / bk_blp   the sparse rows by backward level (over the U
                             entries in sparse columns)
          bk_uoff[p]         for an L entry p = (i, k) with k a sparse row:
                             where the targets of its update start in bk_tgt
          bk_tgt             per L entry (i, k), per U entry (k, j) of row k
                             in order: the place of (i, j) -- an index into
                             the LU values (>= 0) or -1 - its index in S
          bk_jt[e]           the place of Jacobian entry e, the same way
          bk_l21e[i - BK_M]  the end of dense row i's sparse-column L entries
          bk_sk / bk_sp / bk_sl  the Schur complement pivot by pivot: step
                             s eliminates with sparse row bk_sk[s] the dense
                             rows' L entries bk_sl[bk_sp[s] .. bk_sp[s+1])
                             (their places, in row order); bk_st
                             [bk_so[s] .. bk_so[s+1]) the step's update
                             targets, entry by entry then U entry by U
                             entry (bk_tgt in step order)
          bkl_*              the same Schur complement by levels: a step
                             joins the level above every earlier step that
                             writes one of its L entries. Level L divides
                             its L entries bkl_lpl[bkl_lp[L] .. bkl_lp[L+1])
                             by their pivots (rows bkl_lk), then updates its
                             targets bkl_tgt[bkl_tp[L] .. bkl_tp[L+1]), each
                             target t by its contributions bkl_cl / bkl_cu
                             [bkl_cp[t] .. bkl_cp[t+1]) (the places of l
                             and u) in step order: per target the
                             operations and their order are the steps'
          d_bk_hnuc          H nuclei per species (the terms of Hnuclei_)"""
        w = self.w
        D = min(self.BK_DMAX, n)
        m = n - D
        LD = D + 1 if D % 2 == 0 else D
        code = lambda i, j: (pos[(i, j)] if (i < m or j < m)
                             else -1 - ((i - m) * LD + (j - m)))
        lf = [0] * n
        for i in range(m):
            ks = ci[rp[i]:di[i]]
            lf[i] = 1 + max(lf[k] for k in ks) if ks else 0
        nlf = (max(lf[:m]) + 1) if m else 0
        frow = sorted(range(m), key=lambda i: (lf[i], i))
        flp = [0] * (nlf + 1)
        for i in range(m):
            flp[lf[i] + 1] += 1
        for L in range(nlf):
            flp[L + 1] += flp[L]
        lb = [0] * n
        for i in range(m - 1, -1, -1):
            js = [j for j in ci[di[i] + 1:rp[i + 1]] if j < m]
            lb[i] = 1 + max(lb[j] for j in js) if js else 0
        nlb = (max(lb[:m]) + 1) if m else 0
        brow = sorted(range(m), key=lambda i: (lb[i], i))
        blp = [0] * (nlb + 1)
        for i in range(m):
            blp[lb[i] + 1] += 1
        for L in range(nlb):
            blp[L + 1] += blp[L]
        uoff = [-1] * len(ci)
        tgt = []
        l21e = []
        for i in range(n):
            for p in range(rp[i], di[i]):
                k = ci[p]
                if k >= m:
                    continue
                uoff[p] = len(tgt)
                for q in range(di[k] + 1, rp[k + 1]):
                    tgt.append(code(i, ci[q]))
            if i >= m:
                e = rp[i]
                while e < rp[i + 1] and ci[e] < m:
                    e += 1
                l21e.append(e)
        cols = {}
        for i in range(m, n):
            for p in range(rp[i], l21e[i - m]):
                cols.setdefault(ci[p], []).append(p)
        sk = sorted(cols)
        sp_, sl, so, st = [0], [], [0], []
        for k in sk:
            sl += cols[k]
            sp_.append(len(sl))
            nq = rp[k + 1] - di[k] - 1
            for p in cols[k]:
                st += tgt[uoff[p]:uoff[p] + nq]
            so.append(len(st))
        # the Schur steps by levels (a step reads its L entries; it must
        # follow every earlier step that writes one of them)
        nsk = len(sk)
        reads = [set(sl[sp_[t]:sp_[t + 1]]) for t in range(nsk)]
        writer = {}
        lvl = [0] * nsk
        for t in range(nsk):
            lv = 0
            for pl in reads[t]:
                if pl in writer:
                    lv = max(lv, writer[pl] + 1)
            lvl[t] = lv
            for x in st[so[t]:so[t + 1]]:
                if x >= 0:
                    writer[x] = max(writer.get(x, -1), lv)
        nsl = (max(lvl) + 1) if nsk else 0
        lpl, lk, lp = [], [], [0]
        tgt_l, tp, cp, cl, cu = [], [0], [0], [], []
        for L in range(nsl):
            contrib = {}
            order = []
            for t in range(nsk):
                if lvl[t] != L:
                    continue
                k = sk[t]
                q0 = di[k] + 1
                nq = rp[k + 1] - q0
                ents = sl[sp_[t]:sp_[t + 1]]
                for pl in ents:
                    lpl.append(pl)
                    lk.append(k)
                for c, pl in enumerate(ents):
                    for x in range(nq):
                        tg = st[so[t] + c * nq + x]
                        if tg not in contrib:
                            contrib[tg] = []
                            order.append(tg)
                        contrib[tg].append((pl, q0 + x))
            lp.append(len(lpl))
            for tg in order:
                tgt_l.append(tg)
                for pl, q in contrib[tg]:
                    cl.append(pl)
                    cu.append(q)
                cp.append(len(cl))
            tp.append(len(tgt_l))
        inv = {v: key for key, v in pos.items()}
        jt = [code(*inv[q]) for q in jpos]
        self.meta["bk_m"] = m
        self.meta["bk_d"] = D
        w("// the block-per-cell LU: sparse rows [0, BK_M), dense block S of the")
        w("// last BK_D rows (row stride BK_LD) in shared memory")
        w("constexpr int BK_M = %d;" % m)
        w("constexpr int BK_D = %d;" % D)
        w("constexpr int BK_LD = %d;" % LD)
        w("constexpr int BK_NLF = %d;" % nlf)
        w("constexpr int BK_NLB = %d;" % nlb)
        w("constexpr int BK_NTGT = %d;" % len(tgt))
        w("constexpr int BK_NSCHUR = %d;  // Schur steps (pivots)" % len(sk))
        self._table("bk_frow", frow or [0])
        self._table("bk_flp", flp)
        self._table("bk_brow", brow or [0])
        self._table("bk_blp", blp)
        self._table("bk_uoff", uoff)
        self._table("bk_tgt", tgt or [0])
        self._table("bk_jt", jt)
        self._table("bk_l21e", l21e or [0])
        self._table("bk_sk", sk or [0])
        self._table("bk_sp", sp_)
        self._table("bk_sl", sl or [0])
        self._table("bk_so", so)
        self._table("bk_st", st or [0])
        w("constexpr int BK_NSL = %d;  // Schur levels" % nsl)
        self._table("bkl_lp", lp)
        self._table("bkl_lpl", lpl or [0])
        self._table("bkl_lk", lk or [0])
        self._table("bkl_tp", tp)
        self._table("bkl_tgt", tgt_l or [0])
        self._table("bkl_cp", cp)
        self._table("bkl_cl", cl or [0])
        self._table("bkl_cu", cu or [0])
        w("#ifdef __CUDACC__")
        w("__device__ const double d_bk_hnuc[NSPEC] = {%s};"
          % ",".join(repr(float(v)) for v in self.natoms_H))
        w("#endif")

    def _rates_depend_on_n(self):
        """whether a rate coefficient depends on the densities (through
        rates_var or the v_* variables it calls): then the species block of
        the analytic Jacobian, taken at fixed k, is not the exact dF/dn"""
        import re
        text = "\n".join(self.lines)
        bodies = {}
        for m in re.finditer(r"KB_HD inline double (v_\w+)\([^)]*\) \{(.*?)\n\}",
                             text, re.S):
            bodies[m.group(1)] = m.group(2)
        direct = re.compile(r"n\[|\w+_\(n\)")

        def dep(body, seen):
            if direct.search(body):
                return True
            for v in set(re.findall(r"\b(v_\w+)\(", body)) - seen:
                if v in bodies and dep(bodies[v], seen | {v}):
                    return True
            return False
        m = re.search(r"inline void rates_var\(.*?\n\}", text, re.S)
        body = m.group(0).split("{", 1)[1] if m else ""
        body = body.replace("(void)n;", "")
        return dep(body, set())

    # the reference's thermal term lists (runtime/core/solve_cell.hpp:
    # 206-257): name, the generator's flag, and the expression this
    # header evaluates it with (None: not emitted here)
    HEAT_TERMS = [("CUSTOM", None, None), ("CR", "heat_CR", None),
                  ("CHEM", "heat_chem", "heating_chem(T, n, k)"),
                  ("DH", "heat_dH", None),
                  ("COMPRESS", "heat_compress",
                   "ntot_(n) * kbc::boltzmann_erg * T / p.tff"),
                  ("VISCOUS", "heat_visc", None),
                  ("PHOTODUST", "heat_photoDust", None),
                  ("PHOTODUSTNET", "heat_netPhotoDust", None),
                  ("PHOTOAV", "heat_photoAv", None), ("PHOTO", "heat_photo", None),
                  ("ZCIE", "heat_ZCIE", None), ("NUCLEAR", "heat_nuclear", None)]
    COOL_TERMS = [("CUSTOM", None, None),
                  ("ATOMIC", "cool_atomic",
                   "cooling_Atomic(T, n) + cooling_recomb_(T, n, p)"),
                  ("H2", "cool_H2", "cooling_H2(T, n) * h2_opacity_(n)"),
                  ("HD", "cool_HD", None), ("MOL", "cool_mol", None),
                  ("Z", "cool_Z", None), ("Z_CIE", "cool_ZCIE", None),
                  ("Z_EXTENDED", "cool_Zext", None), ("FLOOR", "cooling_floor", None),
                  ("CHEM", "cool_chem", "cooling_chem(n, k)"),
                  ("COMPTON", "cool_compton", None), ("CIE", "cool_CIE", None),
                  ("EXPANSION", "cool_expansion", None),
                  ("CONT", "cool_cont", "cooling_Continuum(T, n)"),
                  ("FF", "cool_ff", None), ("DH", "cool_dH", None),
                  ("DUST", "cool_dust", None), ("DUSTTAB", "cool_dustTab", None),
                  ("DUSTBINS", "cool_dust_bins", None)]

    def emit_interface(self):
        """what the reference's interface reports about a network beyond
        the solve (its query functions): reaction labels, the active
        thermal terms one by one, reaction fluxes, the metallicity
        scaling, the column-density estimate and the photo reactions"""
        w = self.w
        net, gen = self.net, self.gen
        th = gen.thermal
        nrea = len(net.reactions)

        def label(rx):  # the equation, plus the T range of a piece
            s = rx["eq"]
            if rx.get("trange"):
                s += " [%s, %s]" % tuple(self.num(v) for v in rx["trange"])
            return s.replace("\\", "\\\\").replace('"', '\\"')
        w("// reaction labels: the equation, and the T range of a piece")
        w("inline const char* const reaction_names[%d] = {%s};"
          % (max(nrea, 1), ", ".join('"%s"' % label(rx) for rx in net.reactions)))
        # the thermal terms, active ones only, in the reference's order
        heats = [(nm, e) for nm, f, e in self.HEAT_TERMS if f and th.get(f)]
        cools = [(nm, e) for nm, f, e in self.COOL_TERMS if f and th.get(f)]
        for nm, e in heats + cools:
            if e is None:
                raise NotImplementedError("thermal term %s" % nm)
        w("constexpr int NHEAT = %d;" % len(heats))
        w("constexpr int NCOOL = %d;" % len(cools))
        w("inline const char* const heat_names[%d] = {%s};"
          % (max(len(heats), 1), ", ".join('"%s"' % nm for nm, _ in heats) or '""'))
        w("inline const char* const cool_names[%d] = {%s};"
          % (max(len(cools), 1), ", ".join('"%s"' % nm for nm, _ in cools) or '""'))
        w("// the thermal terms one by one [erg cm^-3 s^-1] at the thermal")
        w("// temperature T with the rates k: H[NHEAT], C[NCOOL] in the order")
        w("// of heat_names / cool_names (their sums are thermal_dTdt's)")
        w("KB_HD inline void thermal_terms(double T, const double* n, "
          "const double* k, const Params& p, double* H, double* C) {")
        w("  (void)T; (void)n; (void)k; (void)p; (void)H; (void)C;")
        for j, (_, e) in enumerate(heats):
            w("  H[%d] = %s;" % (j, e))
        for j, (_, e) in enumerate(cools):
            w("  C[%d] = %s;" % (j, e))
        w("}")
        # reaction fluxes
        w("// reaction fluxes k prod(n) [cm^-3 s^-1], fl[NREA]")
        w("KB_HD inline void reaction_fluxes(const double* n, const double* k, "
          "double* fl) {")
        for rx in net.reactions:
            i = rx["id"] - 1
            w("  fl[%d] = %s;" % (i, "*".join(["k[%d]" % i]
                                              + [self.den(s) for s in self._kin(rx)])))
        w("}")
        for rx in net.reactions:
            if rx.get("qeff") or rx.get("nuclear"):
                raise NotImplementedError("qeff / nuclear reactions")
        # metallicity scaling (legacy krome_scale_Z): the neutral atomic
        # metals at n_H 10^(Z + log10(n/n_H)_sun), Asplund+09
        try:
            solar = gen.load_solar()
        except FileNotFoundError:
            solar = {}
        metals = [s for s in self.species if s in solar and s not in ("H", "He")]
        w("// the neutral atomic metals (%s) at n_H 10^(Z + log10(n/n_H)_sun)"
          % (", ".join(metals) or "none"))
        w("// of the Asplund+09 photospheric abundances, floored at 1e-40")
        w("KB_HD inline void scale_Z(double* n, double Z) {")
        w("  (void)n; (void)Z;")
        if metals and "H" in self.species:
            w("  const double Htot = Hnuclei_(n);")
            for m in metals:
                w("  n[IDX_%s] = std::fmax(Htot * std::pow(10.0, Z + (%s)), 1e-40);"
                  % (self.cid(m), self.num(solar[m])))
        w("}")
        # the column density of a number density (radiation.num2col)
        if getattr(gen, "num2col", "default") not in ("default", None, ""):
            raise NotImplementedError("num2col %s" % gen.num2col)
        w("// the column density [cm^-2] of a number density x [cm^-3]")
        w("// (the default estimator: 1.87e21 (x / 1e3)^(2/3))")
        w("KB_HD inline double num2col_(double x) {")
        w("  return 1.87e21 * std::pow(std::fmax(x, 1e-40) * 1e-3, 2.0/3.0);")
        w("}")
        # the H nuclei column N(H) + N(H+) + 2 N(H2) of those estimates
        terms = [("" if sp != "H2" else "2.0 * ") + "num2col_(n[IDX_%s])" % self.cid(sp)
                 for sp in ("H", "H+", "H2") if sp in self.idx]
        w("KB_HD inline double NH_col_(const double* n) {")
        w("  (void)n;")
        w("  return %s;" % (" + ".join(terms) or "0.0"))
        w("}")
        # photo reactions (their rates need a photon field)
        photo = []
        for rx in net.reactions:
            if rx["rate"]["kind"] != "photo":
                continue
            if rx["rate"]["xsec"]["kind"] == "h2pd":
                raise NotImplementedError("h2pd photo channels")
            ph = gen.resolve_photo(rx)
            ph["ch"] = len(photo)
            ph["shield"] = rx["rate"].get("shield")
            if ph["shield"]:
                raise NotImplementedError("shielded photo rates")
            photo.append(ph)
        if any(rx.get("lw") for rx in net.reactions):
            raise NotImplementedError("J_LW rates")
        m = len(photo)
        assert m == len(self.photo_rx)
        w("constexpr int NLW = 0;")
        w("inline const int photo_reaction_[%d] = {%s};"
          % (max(m, 1), ", ".join(str(p["i"]) for p in photo) or "-1"))
        w("inline const int photo_reactant_[%d] = {%s};"
          % (max(m, 1), ", ".join("IDX_" + self.cid(p["reactant"]) for p in photo)
             or "-1"))
        w("inline const double photo_pdiss_[%d] = {%s};"
          % (max(m, 1), ", ".join(self.num(p["rx"].get("pdiss", 1.0)) for p in photo)
             or "1.0"))
        w("// the photoelectron deposit (E - Eth) of each photo rate: none for")
        w("// the Solomon process (line pumping)")
        w("inline const bool photo_deposit_[%d] = {%s};"
          % (max(m, 1), ", ".join("false" if gen.is_solomon(p["rx"]) else "true"
                                  for p in photo) or "true"))
        w("inline const double photo_Emin_[%d] = {%s};"
          % (max(m, 1), ", ".join(self.num(p["Emin"]) for p in photo) or "0.0"))
        w("inline const double photo_Emax_[%d] = {%s};"
          % (max(m, 1), ", ".join(self.num(p["Emax"] if p["Emax"] is not None
                                           else math.inf) for p in photo)
             or "0.0"))
        for p in photo:
            if p.get("edep") or "binned" in p:
                raise NotImplementedError("inner-shell deposits / binned lines")
        # the cross sections sigma_r(E) [cm^2] on the host (the photon bins'
        # averages are built there), rendered by the reference generator's
        # own photo emitter with its tables inline
        if m:
            lines = []
            gen.DATA_THRESHOLD = 1 << 30
            gen.emit_photo(lines.append, photo)
            body = "\n".join(lines)
            body = body.replace("constants::", "kbc::")
            # keep the cross sections, drop the generator's runtime tables
            body = body.split("\nconstexpr int NPHOTO")[0]
            w("// ---- host: the photo cross sections (photon-bin setup) ----")
            w("namespace kbxs {")
            if "H2_sigmaLW" in body:
                # the H2 Lyman-Werner cross section of legacy KROME's
                # H2_sigmaLW (reference runtime/core/h2_shielding.hpp:96-120):
                # the ortho/para-weighted (3:1) sum of the Lyman and Werner
                # band fits of the v = 0 and v = 1 levels, log10 sigma linear
                # or cubic-quintic in E over each band's range
                for ln in (
                    "inline double H2_sigmaLW(double E) {",
                    "  auto band = [](double lg) { return 1e-18 * std::pow(10.0, lg); };",
                    "  double l0 = 0.0, w0 = 0.0, l1 = 0.0, w1 = 0.0;",
                    "  if (E > 14.675 && E < 16.820) l0 = band(15.1289 - 1.05139 * E);",
                    "  else if (E > 16.820 && E < 17.6)",
                    "    l0 = band(-31.41 + 1.8042e-2 * E * E * E - 4.2339e-5 * std::pow(E, 5.0));",
                    "  if (E > 14.675 && E < 17.7) w0 = band(13.5311 - 0.9182618 * E);",
                    "  if (E > 14.159 && E < 15.302) l1 = band(12.0218406 - 0.819429 * E);",
                    "  else if (E > 15.302 && E < 17.2) l1 = band(16.04644 - 1.082438 * E);",
                    "  if (E > 14.159 && E < 17.2) w1 = band(12.87367 - 0.85088597 * E);",
                    "  const double para = 1.0 / (3.0 + 1.0);",
                    "  return para * (l0 + w0) + (1.0 - para) * (l1 + w1);",
                    "}"):
                    w(ln)
            w(body)
            w("inline double (*const photo_xsec[%d])(double) = {%s};"
              % (m, ", ".join("photo_xsec_%d" % p["ch"] for p in photo)))
            w("inline double (*const photo_xsec_int[%d])(double, double) = {%s};"
              % (m, ", ".join(("photo_xsec_int_%d" % p["ch"]) if "table" in p
                              else "nullptr" for p in photo)))
            w("}  // namespace kbxs")
        else:
            w("namespace kbxs {  // no photo reactions")
            w("inline double (*const photo_xsec[1])(double) = {nullptr};")
            w("inline double (*const photo_xsec_int[1])(double, double) = {nullptr};")
            w("}  // namespace kbxs")
        w("")
        self.photo = photo

    def emit_tail(self):
        th = self.gen.thermal
        any_thermal = any(th.get(f) for f in th if f.startswith(("cool_", "heat_")))
        self.w("constexpr bool HAS_THERMAL_TERMS = %s;"
               % ("true" if any_thermal else "false"))
        self.w("// a rate coefficient depends on the densities (the species block")
        self.w("// of jac_stoich, taken at fixed k, is then not the exact dF/dn)")
        self.w("constexpr bool RATES_DEPEND_ON_N = %s;"
               % ("true" if self._rates_depend_on_n() else "false"))
        self.w("}  // namespace kbnet")

    def run(self):
        self.emit_head()
        self.emit_physics()
        self.emit_vars()
        self.emit_surface()
        self.emit_rates()
        self.emit_rhs()
        self.emit_jac()
        if len(self.species) <= LARGE_NSPEC:
            self.emit_jac_dk()
        self.emit_thermal()
        self.emit_lnk_vjp()
        self.emit_interface()
        if len(self.species) > LARGE_NSPEC:
            self.emit_rate_parts()
            self.emit_sparse()
        self.emit_tail()
        return outline_math("\n".join(self.lines) + "\n")


def outline_math(text):
    """route the special functions of the emitted code through kb_common.h's
    wrappers (out of line on the device: one copy of each math routine
    instead of one per call site)"""
    text = re.sub(r"(?<![\w:])(?:std::)?(exp|log10|log|pow)\(", r"kb_\1(", text)
    return text.replace("kb_pow(10.0, ", "kb_exp10(")


def emit(key):
    import json
    em = Emitter(key, NETWORKS[key])
    text = em.run()
    OUTDIR.mkdir(parents=True, exist_ok=True)
    out = OUTDIR / ("net_%s.h" % key)
    out.write_text(text)
    em.meta["nrea_fixed"] = em.nfixed
    (OUTDIR / ("net_%s.json" % key)).write_text(
        json.dumps(em.meta, indent=1) + "\n")
    return out


def main(argv):
    global _REFERENCE
    if "--reference" in argv:
        i = argv.index("--reference")
        _REFERENCE = argv[i + 1]
        argv = argv[:i] + argv[i + 2:]
    keys = argv or list(NETWORKS)
    for k in keys:
        print("wrote", emit(k))


if __name__ == "__main__":
    main(sys.argv[1:])
