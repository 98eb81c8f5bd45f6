// kppcu -- KPP mechanism compiler for the B200 batched Rosenbrock engine.
//
// Data model of a parsed mechanism.  kppcu reads the KPP mechanism language
// (.kpp/.def/.spc/.eqn; the language of src/scan.l + src/scan.y), derives the
// species order and the sparse LU pattern exactly as the reference generator
// does (src/kpp.c:113-403, src/gen.c:331-356), and emits the mechanism's
// rate constants, ODE function, sparse Jacobian, unrolled no-pivot sparse LU
// and triangular solves as CUDA device code for sm_100a.
#pragma once

#include <map>
#include <string>
#include <vector>

namespace kppcu {

enum SpeciesType { SPC_DUMMY = 0, SPC_VAR = 1, SPC_FIX = 2 };
enum RateKind { RATE_NUMBER = 0, RATE_EXPRESSION = 1, RATE_PHOTO = 2 };

struct Species {
  std::string name;
  int type = SPC_DUMMY;
  std::string ival;  // initial value text from #INITVALUES ("" = default)
};

struct Reaction {
  RateKind kind = RATE_EXPRESSION;
  std::string rate;   // rate text, whitespace-free (RATE tokens concatenated)
  float number = 0;   // value of a RATE_NUMBER rate, held as float like KPP
  std::string tag;
};

// Whole mechanism.  Species "codes" are indices into `table` in declaration
// order; `order` lists the codes that take part in equations, in the order
// of first appearance (the reference's Code[] array before reordering).
struct Mechanism {
  std::string root;  // model name used for file names
  std::vector<Species> table;
  std::vector<int> order;            // slot -> species code
  std::map<int, int> slot_of_code;   // species code -> slot
  std::vector<char> reactive;        // per slot: appears on a left-hand side
  // Stoichiometry per slot and reaction, accumulated in float like KPP.
  std::vector<std::vector<float>> left, right, net;
  std::vector<Reaction> reactions;

  // Options and inline code.
  std::map<std::string, std::string> inline_code;  // context -> code
  std::string language = "CUDA";
  std::string integrator;
  bool reorder = true;
  bool use_double = true;
  bool eqntags = false;
  double cfactor = 1.0;
  std::string var_default = "0.", fix_default = "0.";
  std::vector<std::string> warnings;
  int errors = 0;

  // Filled by the structure pass.
  int nvar = 0, nfix = 0, nspec = 0, nvaract = 0;
  std::vector<int> spc_slot;                 // final species index -> slot
  std::vector<std::vector<char>> jstruct;    // [nvar][nvar] Jacobian pattern
  std::vector<std::vector<char>> lustruct;   // [nvar][nvar] after LU fill
  std::vector<int> lu_irow, lu_icol, lu_crow, lu_diag;
  int nonzero = 0, lu_nonzero = 0;

  int find_species(const std::string& name) const;  // code or -1
  int slot_for(int code);                           // allocate on first use
  int nreact() const { return (int)reactions.size(); }
};

// Front end: parse a mechanism file (with includes); search paths are the
// file's own directory, $KPP_HOME/models and $KPP_HOME/int.
bool parse_mechanism(const std::string& path, const std::string& kpp_home, Mechanism& m);

// Structure pass: species ordering, Jacobian and LU sparsity.
void build_structure(Mechanism& m);

// CUDA emitter: writes <out_prefix>.cuh
bool emit_cuda(const Mechanism& m, const std::string& out_prefix);

// Host files: <out_prefix>_host.h (species map of the C ABI) and
// <out_prefix>_Parameters.h (sizes and indices for host models in C).
bool emit_host(const Mechanism& m, const std::string& out_prefix);

}  // namespace kppcu
