/*
 * fn_io.cpp -- the reference's file formats and run flow on top of the C ABI
 * (host code).
 *
 * Parsing follows SimulationManager.cpp function by function: the first line
 * whose first token is the command wins (TextParser::ScanText,
 * TextParser.h:21-38), repeated commands ('type', 'pair', 'output_type',
 * 'output_data', 'modif_*', 'restart_*') are read in file order, numbers go
 * through std::stod / std::stoi / std::stof exactly where the reference uses
 * them.  See include/fibrenet_io.h for the compat / strict differences.
 */
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/fibrenet.h"
#include "../../include/fibrenet_io.h"

struct fn_input {
    fn_settings settings{};
    std::vector<std::string> type_names;
    std::map<std::string, int> type_id;
    std::vector<int> pair_kind;
    std::vector<double> pair_raw;
    std::vector<int> type, tag, loc_id;
    std::vector<double> radius, mass, pos, vel, vel_old, force, img, skin;
    std::vector<int> s_type, s_tag, s_p1, s_p2;
    std::vector<double> s_rest, s_k, s_c1, s_c2, s_damp;
    std::vector<int> a_type, a_tag, a_b1, a_b2, a_b3, a_s1, a_s2;
    std::vector<double> a_theta0, a_k;
    std::vector<int> export_types;
    fn_run_info info{};
    std::string stem;
};

namespace {

using Lines = std::vector<std::vector<std::string>>;

struct Err {
    std::string msg;
};

[[noreturn]] void fail(const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    throw Err{buf};
}

bool read_lines(const std::string& path, Lines& out) {
    std::ifstream f(path);
    if (!f.is_open()) return false;
    std::string line;
    out.clear();
    while (std::getline(f, line)) {
        std::istringstream iss(line);
        std::vector<std::string> toks;
        std::string t;
        while (iss >> t) toks.push_back(t);
        out.push_back(std::move(toks));
    }
    return true;
}

/* TextParser::ScanText: index + 1 of the first line at or after `start`
   whose first token is `key`, and its tokens; -1 when there is none. */
int scan(const Lines& text, const char* key, std::vector<std::string>& tokens, int start) {
    tokens.clear();
    if (start < 0) return -1;
    for (int i = start; i < (int)text.size(); ++i)
        if (!text[i].empty() && text[i][0] == key) {
            tokens = text[i];
            return i + 1;
        }
    return -1;
}

double to_d(const std::string& s, int line) {
    try {
        return std::stod(s);
    } catch (...) {
        fail("line %d: '%s' is not a number", line, s.c_str());
    }
}

int to_i(const std::string& s, int line) {
    try {
        return std::stoi(s);
    } catch (...) {
        fail("line %d: '%s' is not an integer", line, s.c_str());
    }
}

float to_f(const std::string& s, int line) {
    try {
        return std::stof(s);
    } catch (...) {
        fail("line %d: '%s' is not a number", line, s.c_str());
    }
}

/* LoadGlobalForceInfo, SimulationManager.cpp:644-673 */
void global_forces(const Lines& t, fn_input& in) {
    std::vector<std::string> tk;
    int l;
    if ((l = scan(t, "gravity", tk, 0)) > 0) {
        if (tk.size() != 4) fail("line %d: 'gravity' needs three values", l);
        for (int a = 0; a < 3; ++a) in.settings.gravity[a] = to_d(tk[1 + a], l);
    }
    if ((l = scan(t, "damping", tk, 0)) > 0) {
        if (tk.size() != 2) fail("line %d: 'damping' needs one value", l);
        in.settings.damping = to_d(tk[1], l);
    }
}

/* LoadSolverInfo, SimulationManager.cpp:681-819 */
void solver(const Lines& t, fn_input& in, bool strict) {
    std::vector<std::string> tk;
    int l;
    if ((l = scan(t, "step", tk, 0)) <= 0) fail("required command 'step' is missing");
    if (tk.size() != 2) fail("line %d: 'step' needs one value", l);
    in.settings.dt = to_d(tk[1], l);
    if (!(in.settings.dt > 0.0)) fail("line %d: 'step' must be positive", l);
    if ((l = scan(t, "lambda", tk, 0)) > 0) {
        if (tk.size() != 2) fail("line %d: 'lambda' needs one value", l);
        in.settings.lambda = to_d(tk[1], l);
        if (!(in.settings.lambda > 0.0)) fail("line %d: 'lambda' must be positive", l);
    } else {
        if (!strict) fail("required command 'lambda' is missing (SimulationManager.cpp:716-719)");
        in.settings.lambda = 0.5;
    }
    if ((l = scan(t, "run", tk, 0)) <= 0) fail("required command 'run' is missing");
    if (tk.size() != 2) fail("line %d: 'run' needs one value", l);
    in.info.run_steps = to_i(tk[1], l);
    if (in.info.run_steps < 0) fail("line %d: 'run' must not be negative", l);
    in.info.minimize_steps = 0;
    if ((l = scan(t, "minimize_steps", tk, 0)) > 0) {
        if (tk.size() != 2) fail("line %d: 'minimize_steps' needs one value", l);
        in.info.minimize_steps = to_i(tk[1], l);
        if (in.info.minimize_steps < 0) fail("line %d: 'minimize_steps' must not be negative", l);
    }
    if ((l = scan(t, "minimize_substeps", tk, 0)) > 0) {
        if (tk.size() != 2) fail("line %d: 'minimize_substeps' needs one value", l);
        in.info.minimize_substeps = to_i(tk[1], l);
        if (in.info.minimize_substeps < 0 || in.info.minimize_substeps > in.info.minimize_steps)
            fail("line %d: 'minimize_substeps' must lie in [0, minimize_steps]", l);
    } else {
        in.info.minimize_substeps = in.info.minimize_steps > 0 ? in.info.minimize_steps : 0;
    }
    in.info.minimize_reset = 0;
    if ((l = scan(t, "minimize_reset", tk, 0)) > 0) {
        if (tk.size() != 2) fail("line %d: 'minimize_reset' needs one value", l);
        if (tk[1] == "yes")
            in.info.minimize_reset = 1;
        else if (tk[1] != "no")
            fail("line %d: 'minimize_reset' must be yes or no", l);
    }
    if ((l = scan(t, "cutoff", tk, 0)) <= 0) fail("required command 'cutoff' is missing");
    if (tk.size() != 2) fail("line %d: 'cutoff' needs one value", l);
    in.settings.cutoff = to_d(tk[1], l);
    if (!(in.settings.cutoff > 0.0)) fail("line %d: 'cutoff' must be positive", l);
}

/* LoadSimulationBoxInfo, SimulationManager.cpp:2070-2175 */
void box(const Lines& t, fn_input& in, bool strict) {
    std::vector<std::string> tk;
    int l;
    fn_settings& s = in.settings;
    if ((l = scan(t, "box_unit_cell", tk, 0)) <= 0) fail("required command 'box_unit_cell' is missing");
    if (tk.size() != 2) fail("line %d: 'box_unit_cell' needs one value", l);
    s.box_unit_cell = to_d(tk[1], l);
    if (!(s.box_unit_cell > 0.0)) fail("line %d: 'box_unit_cell' must be positive", l);
    if ((l = scan(t, "box_size", tk, 0)) <= 0) fail("required command 'box_size' is missing");
    if (tk.size() != 4) fail("line %d: 'box_size' needs three values", l);
    for (int a = 0; a < 3; ++a) s.box[a] = to_d(tk[1 + a], l);
    for (int a = 0; a < 3; ++a)
        if (s.box[a] < 0.0) fail("line %d: box dimensions must be positive", l);
    for (int a = 0; a < 3; ++a)
        if (s.box[a] / s.box_unit_cell < 3.0)
            fail("line %d: the box must be at least three unit cells along every axis", l);
    if ((l = scan(t, "box_type", tk, 0)) <= 0) fail("required command 'box_type' is missing");
    if (tk.size() != 2) fail("line %d: 'box_type' needs one value", l);
    if (tk[1] == "pbc")
        s.bc_type = 0;
    else if (tk[1] == "finite")
        s.bc_type = 1;
    else
        fail("line %d: 'box_type' must be pbc or finite", l);
    s.grid_update_freq = 8;
    if ((l = scan(t, "grid_update_freq", tk, 0)) > 0) {
        if (tk.size() != 2) fail("line %d: 'grid_update_freq' needs one value", l);
        s.grid_update_freq = to_i(tk[1], l);
        if (s.grid_update_freq <= 0) fail("line %d: 'grid_update_freq' must be positive", l);
    }
    if ((l = scan(t, "box_wall_rep", tk, 0)) > 0) {
        if (tk.size() != 2) fail("line %d: 'box_wall_rep' needs one value", l);
        s.wall_k = to_d(tk[1], l);
        if (s.wall_k < 0.0) fail("line %d: 'box_wall_rep' must not be negative", l);
    } else if (!strict) {
        s.bc_type = 1; /* SimulationManager.cpp:2168 */
    }
    s.periodic_mask = -1;
}

/* LoadTypeAndPairInfo, SimulationManager.cpp:827-970 */
void types_pairs(const Lines& t, fn_input& in) {
    std::vector<std::string> tk;
    int l = 0;
    while ((l = scan(t, "type", tk, l)) != -1) {
        if (tk.size() != 2) fail("line %d: incorrect bead type definition", l);
        if (in.type_id.count(tk[1])) fail("line %d: bead type '%s' redefined", l, tk[1].c_str());
        in.type_id[tk[1]] = (int)in.type_names.size();
        in.type_names.push_back(tk[1]);
    }
    const int nt = (int)in.type_names.size();
    if (nt <= 0) fail("no bead type definitions ('type')");
    in.settings.n_types = nt;
    const int np = nt * (nt - 1) / 2 + nt;
    in.pair_kind.assign(np, 0);
    in.pair_raw.assign(4 * (size_t)np, 0.0);
    std::vector<char> defined(np, 0);
    l = 0;
    while ((l = scan(t, "pair", tk, l)) != -1) {
        if (tk.size() <= 4) fail("line %d: incomplete interaction definition", l);
        auto i1 = in.type_id.find(tk[2]), i2 = in.type_id.find(tk[3]);
        if (i1 == in.type_id.end() || i2 == in.type_id.end())
            fail("line %d: interaction type does not match any defined type", l);
        int t1 = i1->second, t2 = i2->second;
        if (t1 > t2) std::swap(t1, t2);
        const int idx = nt * t1 + t2 - (t1 * (t1 + 1)) / 2;
        int kind, want;
        if (tk[1] == "lj") {
            kind = FN_PAIR_LJ;
            want = 7;
        } else if (tk[1] == "hs") {
            kind = FN_PAIR_HS;
            want = 5;
        } else if (tk[1] == "st") {
            kind = FN_PAIR_ST;
            want = 8;
        } else if (tk[1] == "hsr") {
            kind = FN_PAIR_HSR; /* extension: K k rc */
            want = 7;
        } else {
            fail("line %d: unknown interaction type '%s'", l, tk[1].c_str());
        }
        /* the reference logs a wrong count and stores an uninitialised Pair
           (SimulationManager.cpp:908-936); both modes reject it */
        if ((int)tk.size() != want) fail("line %d: %s interaction needs %d tokens", l, tk[1].c_str(), want);
        in.pair_kind[idx] = kind;
        for (int k = 0; k < 4; ++k) in.pair_raw[4 * (size_t)idx + k] = 4 + k < want ? to_d(tk[4 + k], l) : 0.0;
        defined[idx] = 1;
    }
    for (int i = 0; i < np; ++i)
        if (!defined[i])
            fail("pair list contains undefined interactions: every type-type pair needs a 'pair' line");
}

/* LoadExportInfo, SimulationManager.cpp:979-1091 */
void exports(const Lines& t, fn_input& in) {
    std::vector<std::string> tk;
    int l;
    if ((l = scan(t, "output_file", tk, 0)) <= 0) fail("required command 'output_file' is missing");
    if (tk.size() != 2) fail("line %d: 'output_file' needs one value", l);
    in.stem = tk[1];
    if ((l = scan(t, "output_freq", tk, 0)) <= 0) fail("required command 'output_freq' is missing");
    if (tk.size() != 2) fail("line %d: 'output_freq' needs one value", l);
    in.info.output_freq = to_i(tk[1], l);
    if (in.info.output_freq <= 0) fail("line %d: 'output_freq' must be positive", l);
    if (in.info.output_freq > in.info.run_steps) fail("line %d: 'output_freq' must not exceed 'run'", l);
    l = 0;
    while ((l = scan(t, "output_type", tk, l)) != -1) {
        if (tk.size() != 2) fail("line %d: 'output_type' needs one value", l);
        if (tk[1] == "all") {
            in.export_types.clear();
            for (auto& kv : in.type_id) in.export_types.push_back(kv.second);
        } else {
            auto it = in.type_id.find(tk[1]);
            if (it == in.type_id.end()) fail("line %d: export type does not match any defined type", l);
            bool have = false;
            for (int x : in.export_types) have |= x == it->second;
            if (!have) in.export_types.push_back(it->second);
        }
    }
    if (in.export_types.empty()) fail("no exported bead types ('output_type')");
    l = 0;
    while ((l = scan(t, "output_data", tk, l)) != -1) {
        if (tk.size() != 2) fail("line %d: 'output_data' needs one value", l);
        if (tk[1] == "position")
            in.info.export_position = 1;
        else if (tk[1] == "velocity")
            in.info.export_velocity = 1;
        else if (tk[1] == "force")
            in.info.export_force = 1;
        else if (tk[1] == "all")
            in.info.export_position = in.info.export_velocity = in.info.export_force = 1;
        else
            fail("line %d: unknown 'output_data' value '%s'", l, tk[1].c_str());
    }
    if (!in.info.export_position && !in.info.export_velocity && !in.info.export_force)
        fail("no exported quantity ('output_data')");
}

/* ReadBeadsData, SimulationManager.cpp:1372-1493 */
void beads(const Lines& t, fn_input& in, bool strict) {
    std::vector<std::string> tk;
    int l = 0;
    while ((l = scan(t, "BEAD", tk, l)) != -1) {
        if (tk.size() != 18) fail("model line %d: a BEAD line has 18 fields", l);
        double p[3];
        for (int a = 0; a < 3; ++a) p[a] = to_d(tk[6 + a], l);
        for (int a = 0; a < 3; ++a)
            if (p[a] > in.settings.box[a] || p[a] < 0.0)
                fail("model line %d: bead lies outside the simulation box", l);
        double v[3], f[3], im[3];
        for (int a = 0; a < 3; ++a) v[a] = to_d(tk[9 + a], l);
        for (int a = 0; a < 3; ++a) f[a] = to_d(tk[12 + a], l);
        for (int a = 0; a < 3; ++a) im[a] = to_d(tk[15 + a], l);
        auto it = in.type_id.find(tk[1]);
        if (it == in.type_id.end()) fail("model line %d: bead type does not match any defined type", l);
        in.type.push_back(it->second);
        in.tag.push_back(to_i(tk[2], l));
        in.loc_id.push_back(to_i(tk[3], l));
        const double r = to_d(tk[4], l);
        in.radius.push_back(r);
        in.skin.push_back(r + 0.5);
        in.mass.push_back(to_d(tk[5], l));
        for (int a = 0; a < 3; ++a) {
            in.pos.push_back(p[a]);
            in.vel.push_back(v[a]);
            /* velocity_old.{x,y,z} = velocity.x in the reference (:1405-1407) */
            in.vel_old.push_back(strict ? v[a] : v[0]);
            in.force.push_back(f[a]);
            in.img.push_back(im[a]);
        }
    }
    if (in.type.empty()) fail("the model defines no beads");
}

/* ReadSpringData, SimulationManager.cpp:1501-1583 */
void springs(const Lines& t, fn_input& in, bool strict) {
    std::vector<std::string> tk;
    int l = 0;
    while ((l = scan(t, "SPRING", tk, l)) != -1) {
        if (tk.size() < 2) fail("model line %d: invalid spring", l);
        int type;
        double c1 = 0.0, c2 = 0.0;
        if (tk[1] == "HR") {
            if (tk.size() < 7) fail("model line %d: an HR spring has at least 7 fields", l);
            type = 0;
        } else if (tk[1] == "HR_FL") {
            if (tk.size() != 9) fail("model line %d: an HR_FL spring has 9 fields", l);
            type = 1;
            /* std::stoi in the reference (:1528-1529) */
            c1 = strict ? to_d(tk[7], l) : (double)to_i(tk[7], l);
            c2 = strict ? to_d(tk[8], l) : (double)to_i(tk[8], l);
        } else {
            fail("model line %d: unknown spring type '%s'", l, tk[1].c_str());
        }
        const int nb = (int)in.type.size();
        const int p1 = to_i(tk[3], l), p2 = to_i(tk[4], l);
        if (p1 < 0 || p1 >= nb || p2 < 0 || p2 >= nb) fail("model line %d: spring references a missing bead", l);
        const double rest = to_d(tk[5], l), k = to_d(tk[6], l);
        if (rest < 0.0) fail("model line %d: negative rest length", l);
        if (k < 0.0) fail("model line %d: negative stiffness", l);
        in.s_type.push_back(type);
        in.s_tag.push_back(to_i(tk[2], l));
        in.s_p1.push_back(p1);
        in.s_p2.push_back(p2);
        in.s_rest.push_back(rest);
        in.s_k.push_back(k);
        in.s_c1.push_back(c1);
        in.s_c2.push_back(c2);
        in.s_damp.push_back(0.0);
    }
}

/* ReadAngleData, SimulationManager.cpp:1591-1661 */
void angles(const Lines& t, fn_input& in, bool strict) {
    std::vector<std::string> tk;
    int l = 0;
    while ((l = scan(t, "ANGLE", tk, l)) != -1) {
        if (tk.size() != 10) fail("model line %d: an ANGLE line has 10 fields", l);
        int type;
        if (tk[1] == "HR")
            type = 0;
        else if (tk[1] == "HR_FL")
            type = 1;
        else
            fail("model line %d: unknown angle type '%s'", l, tk[1].c_str());
        const int nb = (int)in.type.size(), ns = (int)in.s_type.size();
        int b[3];
        for (int q = 0; q < 3; ++q) {
            b[q] = to_i(tk[3 + q], l);
            if (b[q] < 0 || b[q] >= nb) fail("model line %d: angle references a missing bead", l);
        }
        const int s1 = to_i(tk[6], l), s2 = to_i(tk[7], l);
        if (type == 1 && (s1 < 0 || s1 >= ns || s2 < 0 || s2 >= ns))
            fail("model line %d: HR_FL angle references a missing spring", l);
        in.a_type.push_back(type);
        in.a_tag.push_back(to_i(tk[2], l));
        in.a_b1.push_back(b[0]);
        in.a_b2.push_back(b[1]);
        in.a_b3.push_back(b[2]);
        in.a_s1.push_back(s1);
        in.a_s2.push_back(s2);
        in.a_theta0.push_back(strict ? to_d(tk[8], l) : (double)to_f(tk[8], l)); /* std::stof, :1637 */
        in.a_k.push_back(to_d(tk[9], l));
    }
}

/* ReadRestartFile, SimulationManager.cpp:1670-1823 */
void restart(const Lines& t, fn_input& in) {
    std::vector<std::string> tk;
    std::string file;
    bool rp = false, rv = false, rf = false;
    int l = 0;
    while ((l = scan(t, "restart_file", tk, l)) != -1) {
        if (tk.size() != 2) fail("line %d: 'restart_file' needs one value", l);
        file = tk[1];
    }
    l = 0;
    while ((l = scan(t, "restart_data", tk, l)) != -1) {
        if (tk.size() != 2) fail("line %d: 'restart_data' needs one value", l);
        if (tk[1] == "position")
            rp = true;
        else if (tk[1] == "velocity")
            rv = true;
        else if (tk[1] == "force")
            rf = true;
        else if (tk[1] == "all")
            rp = rv = rf = true;
        else
            fail("line %d: unknown 'restart_data' value", l);
    }
    if (file.empty()) return;
    Lines r;
    if (!read_lines(file, r)) fail("unable to open restart file %s", file.c_str());
    if (r.empty()) fail("restart file %s is empty", file.c_str());
    const int nb = (int)in.type.size();
    int bi = 0;
    for (size_t q = 0; q < r.size(); ++q) {
        const auto& x = r[q];
        if (x.size() != 13) continue;
        if (bi >= nb) fail("restart file has more beads than the model");
        auto it = in.type_id.find(x[0]);
        if (it == in.type_id.end()) fail("restart file: unknown bead type '%s'", x[0].c_str());
        if (it->second != in.type[bi]) fail("restart file: type of bead %d differs from the model", bi);
        const int ln = (int)q + 1;
        if (rp)
            for (int a = 0; a < 3; ++a) {
                in.pos[3 * bi + a] = to_d(x[1 + a], ln);
                in.img[3 * bi + a] = to_d(x[4 + a], ln);
            }
        if (rv)
            for (int a = 0; a < 3; ++a) {
                in.vel[3 * bi + a] = to_d(x[7 + a], ln);
                in.vel_old[3 * bi + a] = in.vel[3 * bi + a];
            }
        if (rf)
            for (int a = 0; a < 3; ++a) in.force[3 * bi + a] = to_d(x[10 + a], ln);
        ++bi;
    }
    if (bi != nb) fail("restart file holds %d beads, the model %d", bi, nb);
}

/* LoadBeadModifications, SimulationManager.cpp:189-415 */
void bead_modifs(const Lines& t, fn_input& in) {
    std::vector<std::string> tk;
    int l = 0;
    const int nb = (int)in.type.size();
    while ((l = scan(t, "modif_bead", tk, l)) != -1) {
        if (tk.size() <= 4) fail("line %d: 'modif_bead' needs a selection, a property and a value", l);
        int sel, key;
        if (tk[1] == "id")
            sel = 0;
        else if (tk[1] == "tag")
            sel = 1;
        else if (tk[1] == "type")
            sel = 2;
        else
            fail("line %d: 'modif_bead' selection must be id, tag or type", l);
        if (sel == 2) {
            auto it = in.type_id.find(tk[2]);
            if (it == in.type_id.end()) fail("line %d: unknown bead type '%s'", l, tk[2].c_str());
            key = it->second;
        } else {
            key = to_i(tk[2], l);
        }
        auto match = [&](int i) {
            return (sel == 0 && i == key) || (sel == 1 && in.tag[i] == key) || (sel == 2 && in.type[i] == key);
        };
        if (tk[3] == "mass") {
            if (tk.size() != 5) fail("line %d: 'modif_bead ... mass' needs one value", l);
            const double m = to_d(tk[4], l);
            if (m < 0.0) fail("line %d: mass must be zero or positive", l);
            for (int i = 0; i < nb; ++i)
                if (match(i)) in.mass[i] = m;
        } else if (tk[3] == "velocity") {
            if (tk.size() != 7) fail("line %d: 'modif_bead ... velocity' needs three values", l);
            double v[3];
            for (int a = 0; a < 3; ++a) v[a] = to_d(tk[4 + a], l);
            for (int i = 0; i < nb; ++i)
                if (match(i))
                    for (int a = 0; a < 3; ++a) in.vel[3 * i + a] = in.vel_old[3 * i + a] = v[a];
        } else if (tk[3] == "skin_radius") {
            if (tk.size() != 5) fail("line %d: 'modif_bead ... skin_radius' needs one value", l);
            const double s = to_d(tk[4], l);
            for (int i = 0; i < nb; ++i)
                if (match(i)) in.skin[i] = s;
            in.info.has_skin_override = 1;
        } else {
            fail("line %d: unknown 'modif_bead' property '%s'", l, tk[3].c_str());
        }
    }
}

/* LoadSpringModifications, SimulationManager.cpp:423-636 */
void spring_modifs(const Lines& t, fn_input& in) {
    std::vector<std::string> tk;
    int l = 0;
    const int ns = (int)in.s_type.size();
    while ((l = scan(t, "modif_spring", tk, l)) != -1) {
        if (tk.size() <= 4) fail("line %d: 'modif_spring' needs a selection, a property and a value", l);
        int sel;
        if (tk[1] == "id")
            sel = 0;
        else if (tk[1] == "tag")
            sel = 1;
        else
            fail("line %d: 'modif_spring' selection must be id or tag", l);
        const int key = to_i(tk[2], l);
        std::vector<double>* field = nullptr;
        if (tk[3] == "c1")
            field = &in.s_c1;
        else if (tk[3] == "c2")
            field = &in.s_c2;
        else if (tk[3] == "rest_length")
            field = &in.s_rest;
        else if (tk[3] == "stiffness")
            field = &in.s_k;
        else if (tk[3] == "damping")
            field = &in.s_damp; /* read by no kernel */
        else
            fail("line %d: unknown 'modif_spring' property '%s'", l, tk[3].c_str());
        if (tk.size() != 5) {
            /* the reference only logs a malformed stiffness or damping
               change and goes on (SimulationManager.cpp:585-587, 615-617) */
            if (!in.info.strict && (field == &in.s_k || field == &in.s_damp)) continue;
            fail("line %d: 'modif_spring' needs one value", l);
        }
        const double v = to_d(tk[4], l);
        if (v < 0.0) fail("line %d: the value must be zero or positive", l);
        for (int s = 0; s < ns; ++s)
            if ((sel == 0 && s == key) || (sel == 1 && in.s_tag[s] == key)) (*field)[s] = v;
    }
}

void copy_err(const std::string& m, char* err, int err_len) {
    if (err && err_len > 0) {
        std::strncpy(err, m.c_str(), (size_t)err_len - 1);
        err[err_len - 1] = 0;
    }
}

/* ------------------------------------------------------------------ */
/* outputs                                                              */

struct Dumper {
    const fn_input* in;
    std::vector<int> index;        /* exported beads, bead order */
    std::FILE *fpos = nullptr, *fvel = nullptr, *fforce = nullptr;
    float restart_stage = 0.25f;   /* SimulationManager.cpp:1941 */
    ~Dumper() {
        if (fpos) std::fclose(fpos);
        if (fvel) std::fclose(fvel);
        if (fforce) std::fclose(fforce);
    }
};

/* The XYZ frame of DumpData (SimulationManager.cpp:2001-2049): the stream is
   std::fixed with 5 decimals once the first frame has been written. */
void write_frame(std::FILE* f, const Dumper& d, int progress, const std::vector<double>& v) {
    const fn_settings& s = d.in->settings;
    std::fprintf(f, "%zu\nFRAME\t%d\t%.5f\t%.5f\t%.5f\t%.5f\n", d.index.size(), progress, s.dt, s.box[0],
                 s.box[1], s.box[2]);
    for (int i : d.index)
        std::fprintf(f, "%s\t%.5f\t%.5f\t%.5f\n", d.in->type_names[d.in->type[i]].c_str(), v[3 * i],
                     v[3 * i + 1], v[3 * i + 2]);
    std::fflush(f);
}

/* DumpRestartData (SimulationManager.cpp:1855-1928): default stream
   formatting (6 significant digits) in compat mode, exact in strict mode. */
bool write_restart(fn_ctx* ctx, const fn_input& in, int progress) {
    const size_t nb = in.type.size();
    std::vector<double> p(3 * nb), im(3 * nb), v(3 * nb), f(3 * nb);
    if (fn_download(ctx, FN_POSITION, p.data()) || fn_download(ctx, FN_IMAGE, im.data()) ||
        fn_download(ctx, FN_VELOCITY, v.data()) || fn_download(ctx, FN_FORCE, f.data()))
        return false;
    std::FILE* o = std::fopen((in.stem + "_restart.res").c_str(), "w");
    if (!o) return false;
    const char* g = in.info.strict ? "%.17g" : "%g";
    auto num = [&](double x) { std::fprintf(o, "\t"); std::fprintf(o, g, x); };
    std::fprintf(o, "%zu\nFRAME\t%d", nb, progress);
    num(in.settings.dt);
    for (int a = 0; a < 3; ++a) num(in.settings.box[a]);
    std::fprintf(o, "\n");
    for (size_t i = 0; i < nb; ++i) {
        std::fprintf(o, "\t%s", in.type_names[in.type[i]].c_str());
        for (int a = 0; a < 3; ++a) num(p[3 * i + a]);
        for (int a = 0; a < 3; ++a) num(im[3 * i + a]);
        for (int a = 0; a < 3; ++a) num(v[3 * i + a]);
        for (int a = 0; a < 3; ++a) num(f[3 * i + a]);
        std::fprintf(o, "\n");
    }
    std::fclose(o);
    return true;
}

bool dump(fn_ctx* ctx, Dumper& d, int progress) {
    const fn_input& in = *d.in;
    const size_t nb = in.type.size();
    std::vector<double> buf(3 * nb);
    if (in.info.export_position) {
        if (fn_download(ctx, FN_POSITION, buf.data())) return false;
        write_frame(d.fpos, d, progress, buf);
    }
    if (in.info.export_velocity) {
        if (fn_download(ctx, FN_VELOCITY, buf.data())) return false;
        write_frame(d.fvel, d, progress, buf);
    }
    if (in.info.export_force) {
        if (fn_download(ctx, FN_FORCE, buf.data())) return false;
        write_frame(d.fforce, d, progress, buf);
    }
    if (in.info.run_steps > 0 &&
        (static_cast<float>(progress) / static_cast<float>(in.info.run_steps)) > d.restart_stage) {
        d.restart_stage += 0.25f;
        if (!write_restart(ctx, in, progress)) return false;
    }
    return true;
}

}  // namespace

/* ======================================================================== */

extern "C" {

FN_IO_API int fn_input_read(const char* input_path, int strict, fn_input** out, char* err, int err_len) {
    if (!input_path || !out) return FN_ERR_ARG;
    *out = nullptr;
    fn_input* in = new fn_input();
    in->info.strict = strict ? 1 : 0;
    in->settings.skin_ratio = 0.5; /* SimulationManager.cpp:26 */
    try {
        Lines t;
        if (!read_lines(input_path, t)) fail("unable to open input file %s", input_path);
        global_forces(t, *in);
        solver(t, *in, strict != 0);
        box(t, *in, strict != 0);
        types_pairs(t, *in);
        exports(t, *in);
        std::vector<std::string> tk;
        int l;
        if ((l = scan(t, "model_file", tk, 0)) <= 0) fail("the input file names no 'model_file'");
        if (tk.size() != 2) fail("line %d: 'model_file' needs one value", l);
        Lines m;
        if (!read_lines(tk[1], m)) fail("unable to open model file %s", tk[1].c_str());
        if (m.empty()) fail("model file %s is empty", tk[1].c_str());
        beads(m, *in, strict != 0);
        springs(m, *in, strict != 0);
        angles(m, *in, strict != 0);
        restart(t, *in);
        bead_modifs(t, *in);
        spring_modifs(t, *in);
    } catch (const Err& e) {
        copy_err(e.msg, err, err_len);
        delete in;
        return FN_ERR_ARG;
    } catch (const std::bad_alloc&) {
        copy_err("out of host memory", err, err_len);
        delete in;
        return FN_ERR_OOM;
    } catch (const std::exception& e) {
        copy_err(e.what(), err, err_len);
        delete in;
        return FN_ERR_ARG;
    }
    copy_err("", err, err_len);
    *out = in;
    return FN_OK;
}

FN_IO_API void fn_input_free(fn_input* in) { delete in; }

FN_IO_API int fn_input_desc(const fn_input* in, fn_network_desc* d) {
    if (!in || !d) return FN_ERR_ARG;
    std::memset(d, 0, sizeof *d);
    d->settings = in->settings;
    d->pair_kind = in->pair_kind.data();
    d->pair_raw = in->pair_raw.data();
    d->n_beads = (int)in->type.size();
    d->type = in->type.data();
    d->tag = in->tag.data();
    d->loc_id = in->loc_id.data();
    d->radius = in->radius.data();
    d->mass = in->mass.data();
    d->pos = in->pos.data();
    d->vel = in->vel.data();
    d->vel_old = in->vel_old.data();
    d->force = in->force.data();
    d->img = in->img.data();
    d->n_springs = (int)in->s_type.size();
    d->s_type = in->s_type.data();
    d->s_p1 = in->s_p1.data();
    d->s_p2 = in->s_p2.data();
    d->s_rest = in->s_rest.data();
    d->s_k = in->s_k.data();
    d->s_c1 = in->s_c1.data();
    d->s_c2 = in->s_c2.data();
    d->n_angles = (int)in->a_type.size();
    d->a_type = in->a_type.data();
    d->a_b1 = in->a_b1.data();
    d->a_b2 = in->a_b2.data();
    d->a_b3 = in->a_b3.data();
    d->a_s1 = in->a_s1.data();
    d->a_s2 = in->a_s2.data();
    d->a_theta0 = in->a_theta0.data();
    d->a_k = in->a_k.data();
    return FN_OK;
}

FN_IO_API int fn_input_info(const fn_input* in, fn_run_info* out) {
    if (!in || !out) return FN_ERR_ARG;
    *out = in->info;
    return FN_OK;
}

FN_IO_API const double* fn_input_skin(const fn_input* in) { return in ? in->skin.data() : nullptr; }

FN_IO_API const char* fn_input_type_name(const fn_input* in, int t) {
    if (!in || t < 0 || t >= (int)in->type_names.size()) return nullptr;
    return in->type_names[t].c_str();
}

FN_IO_API const char* fn_input_output_stem(const fn_input* in) { return in ? in->stem.c_str() : nullptr; }

static int run_input(const char* input_path, int device, int strict, char* err, int err_len);

/* The Run flow behind a guard: no C++ exception crosses the C ABI. */
FN_IO_API int fn_run_input(const char* input_path, int device, int strict, char* err, int err_len) {
    try {
        return run_input(input_path, device, strict, err, err_len);
    } catch (const std::bad_alloc&) {
        copy_err("out of host memory", err, err_len);
        return FN_ERR_OOM;
    } catch (const std::exception& e) {
        copy_err(e.what(), err, err_len);
        return FN_ERR_ARG;
    }
}

static int run_input(const char* input_path, int device, int strict, char* err, int err_len) {
    fn_input* in = nullptr;
    int rc = fn_input_read(input_path, strict, &in, err, err_len);
    if (rc) return rc;
    fn_config cfg = {device, 64, 128, 1, 0, 0, 0, 0.0, 0};
    fn_ctx* ctx = nullptr;
    auto finish = [&](int code, const std::string& msg) {
        if (!msg.empty()) copy_err(msg, err, err_len);
        if (ctx) fn_destroy(ctx);
        fn_input_free(in);
        return code;
    };
    if ((rc = fn_create(&cfg, &ctx)) != FN_OK) return finish(rc, "no CUDA device");
    fn_network_desc d;
    fn_input_desc(in, &d);
    if ((rc = fn_upload(ctx, 1, &d)) != FN_OK) return finish(rc, fn_last_error(ctx));
    if (in->info.has_skin_override && (rc = fn_set_skin(ctx, in->skin.data())) != FN_OK)
        return finish(rc, fn_last_error(ctx));

    /* InitializeDataDump, SimulationManager.cpp:1099-1145 */
    Dumper dmp;
    dmp.in = in;
    for (size_t i = 0; i < in->type.size(); ++i)
        for (int x : in->export_types)
            if (in->type[i] == x) {
                dmp.index.push_back((int)i);
                break;
            }
    if (dmp.index.empty()) return finish(FN_ERR_ARG, "declared export types not found in the model");
    /* DumpData opens the files in append mode (SimulationManager.cpp:1970-1987) */
    if (in->info.export_position && !(dmp.fpos = std::fopen((in->stem + "_coord.xyz").c_str(), "a")))
        return finish(FN_ERR_ARG, "unable to open " + in->stem + "_coord.xyz");
    if (in->info.export_velocity && !(dmp.fvel = std::fopen((in->stem + "_vel.xyz").c_str(), "a")))
        return finish(FN_ERR_ARG, "unable to open " + in->stem + "_vel.xyz");
    if (in->info.export_force && !(dmp.fforce = std::fopen((in->stem + "_force.xyz").c_str(), "a")))
        return finish(FN_ERR_ARG, "unable to open " + in->stem + "_force.xyz");

    /* MinimizeSystemEnergy, SimulationManager.cpp:111-143 */
    const fn_run_info& ri = in->info;
    if (ri.minimize_steps > 0) {
        if (ri.minimize_reset && (rc = fn_reset_energy(ctx))) return finish(rc, fn_last_error(ctx));
        if (ri.minimize_substeps <= 0) return finish(FN_ERR_ARG, "'minimize_substeps' must be positive");
        const int loops = ri.minimize_steps / ri.minimize_substeps;
        for (int q = 0; q < loops; ++q) {
            if ((rc = fn_step(ctx, ri.minimize_substeps))) return finish(rc, fn_last_error(ctx));
            if (ri.minimize_reset && (rc = fn_reset_energy(ctx))) return finish(rc, fn_last_error(ctx));
        }
    }
    /* Run, SimulationManager.cpp:74-95 */
    int progress = 0;
    if (!dump(ctx, dmp, progress)) return finish(FN_ERR_CUDA, fn_last_error(ctx));
    while (progress < ri.run_steps) {
        const int chunk = (ri.run_steps - progress) < ri.output_freq ? ri.run_steps - progress : ri.output_freq;
        if ((rc = fn_step(ctx, chunk))) return finish(rc, fn_last_error(ctx));
        progress += chunk;
        if (!dump(ctx, dmp, progress)) return finish(FN_ERR_CUDA, fn_last_error(ctx));
        std::fprintf(stderr, "\tSimulation progress: finished %d out of %d simulation steps\n", progress,
                     ri.run_steps);
    }
    if (!write_restart(ctx, *in, progress)) return finish(FN_ERR_CUDA, "unable to write the final restart file");
    return finish(FN_OK, "");
}

}  // extern "C"
