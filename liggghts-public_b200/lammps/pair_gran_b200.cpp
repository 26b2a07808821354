/* pair_style gran/b200 -- see pair_gran_b200.h */
#include "pair_gran_b200.h"

#include <cstring>

#include "b200_args.h"
#include "error.h"
#include "force.h"
#include "lammps.h"
#include "update.h"

using namespace LAMMPS_NS;

PairGranB200::PairGranB200(LAMMPS *lmp) : PairGranProxy(lmp), rolling_cdt_(0), tangential_damping_(1) {}

/* PairGranProxy::settings (src/pair_gran_proxy.cpp:63) after checking that
   the model and its settings are the accelerated ones */
void PairGranB200::settings(int narg, char **arg)
{
  B200::ModelArgs m;
  int i = m.parse_pairs(narg, arg, 0);
  while (i >= 0 && i < narg) {
    const int used = m.parse_setting(narg, arg, i);
    if (!used) {
      m.fail(arg[i], "");
      break;
    }
    i += used;
  }
  if (!m.bad.empty()) {
    std::string msg = "pair_style gran/b200: '" + m.bad + "' is outside the accelerated path (model hertz "
                      "tangential history [rolling_friction cdt] [tangential_damping on|off])";
    error->all(FLERR, msg.c_str());
  }
  rolling_cdt_ = m.rolling_cdt;
  tangential_damping_ = m.tangential_damping;
  PairGranProxy::settings(narg, arg);
  // the reference's own granular fixes and computes look the pair style up
  // by its exact name (force->pair_match("gran", 1), src/fix_contact_history.
  // cpp:218 and others): register under the reference's name
  delete [] force->pair_style;
  force->pair_style = new char[5];
  strcpy(force->pair_style, "gran");
  // the default integrator is created before the command line's suffix is
  // known (src/update.cpp:99); with "-sf b200" / "suffix b200" in force the
  // run becomes device-resident: run_style verlet -> verlet/b200
  if (lmp->suffix_enable && lmp->suffix && !strcmp(lmp->suffix, "b200") && update->integrate_style &&
      !strcmp(update->integrate_style, "verlet")) {
    char style[] = "verlet";
    char *args[] = {style};
    update->create_integrate(1, args, lmp->suffix);
  }
}
