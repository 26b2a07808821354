/* b200_args.h -- shared argument checks of the b200 suffix styles.
 *
 * The b200 styles accept exactly the input grammar of the granular path the
 * device runs (pair_style gran / fix wall/gran model grammar, src/
 * contact_models.cpp:158 Factory::select_model and the model settings of
 * src/normal_model_hertz.h:88-96) and reject everything else through
 * error->all, naming the keyword, so an input script outside that path fails
 * loudly instead of silently running another model.
 */
#ifndef LMP_B200_ARGS_H
#define LMP_B200_ARGS_H

#include <cstring>
#include <string>

namespace LAMMPS_NS {
namespace B200 {

/* the contact-model part of a pair_style gran / fix wall/gran argument list:
 * pairs "model hertz", "tangential history", "rolling_friction cdt|off",
 * "cohesion off", "surface default" in any order, then the model settings
 * "tangential_damping on|off".  Returns the index after the model pairs (the
 * settings are parsed by parse_settings, wherever they stand). */
struct ModelArgs {
    int rolling_cdt = 0;
    int tangential_damping = 1;
    bool have_model = false, have_tangential = false;
    std::string bad;   // first keyword outside the accelerated path

    int parse_pairs(int narg, char **arg, int i)
    {
        while (i + 1 < narg) {
            const char *k = arg[i], *v = arg[i + 1];
            if (!strcmp(k, "model")) {
                if (strcmp(v, "hertz")) return fail(k, v);
                have_model = true;
            } else if (!strcmp(k, "tangential")) {
                if (strcmp(v, "history")) return fail(k, v);
                have_tangential = true;
            } else if (!strcmp(k, "rolling_friction")) {
                if (!strcmp(v, "cdt")) rolling_cdt = 1;
                else if (!strcmp(v, "off")) rolling_cdt = 0;
                else return fail(k, v);
            } else if (!strcmp(k, "cohesion")) {
                if (strcmp(v, "off")) return fail(k, v);
            } else if (!strcmp(k, "surface")) {
                if (strcmp(v, "default")) return fail(k, v);
            } else {
                break;
            }
            i += 2;
        }
        if (bad.empty() && !(have_model && have_tangential)) bad = "model hertz tangential history (required)";
        return i;
    }
    /* one model setting at arg[i]; returns the count consumed (0: not one) */
    int parse_setting(int narg, char **arg, int i)
    {
        if (i + 1 < narg && !strcmp(arg[i], "tangential_damping")) {
            if (!strcmp(arg[i + 1], "on")) tangential_damping = 1;
            else if (!strcmp(arg[i + 1], "off")) tangential_damping = 0;
            else fail(arg[i], arg[i + 1]);
            return 2;
        }
        return 0;
    }
    int fail(const char *k, const char *v)
    {
        if (bad.empty()) bad = std::string(k) + " " + v;
        return -1;
    }
};

}  // namespace B200
}  // namespace LAMMPS_NS

#endif
