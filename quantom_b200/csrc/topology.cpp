// Real-topology input (host C++): a GROMACS conf.gro + topol.top and CHARMM
// parameter files -> the reference's box arrays (force field, compounds,
// bridges, solvents), ready for lima_load_*.  It replaces the reference's
// three-stage input path with one pass in memory:
//   1. LIMA_ForcefieldMaker (ForcefieldMerger.h:9-170, ForcefieldTypes.h,
//      LIMA_ForcefieldMaker.cpp:16-146): CHARMM NONBONDED / BONDS / ANGLES /
//      DIHEDRALS merged into typed tables, the conf's atom names mapped onto
//      non-bonded types by dropping trailing characters until a type exists,
//      and every topology bond, angle and dihedral given the parameters of the
//      best prefix-matching ("likeness") type entry;
//   2. ForceFieldMaker::buildForcefield (Forcefield.cu:10-218): the per-atom
//      type ids and per-term parameters the compounds are built from;
//   3. CompoundBuilder::buildMolecule (CompoundBuilder.cpp:7-463) and
//      BoxBuilder::addSingleMolecule / solvateBox (BoxBuilder.cu:42-218):
//      residues packed into compounds of at most 64 particles, a bridge
//      between consecutive compounds for terms that span them, LJ exclusions
//      between every pair of atoms sharing a term, the molecule centred in the
//      box and the conf's water oxygens added as solvents where there is room.
// The reference passes its tables between the stages as text files written
// with std::to_string (six decimals) and read back with stof; here every value
// takes the same round trips (rt below), so the parameters come out as the
// reference's simulations see them.  The reference draws solvent velocity
// directions from the C library's random(); here they are uniform on the
// sphere from a seeded generator, with the reference's speed sqrt(3 R T / M).
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "lima_abi.h"

struct lima_topology {
    std::string err;
    lima_forcefield ff{};
    int n_types = 0;
    std::vector<lima_compound> comps;
    std::vector<lima_compound_state> states;
    std::vector<lima_compound_bridge_compact> bridges;
    std::vector<lima_solvent> sols;
};

namespace {

struct BuildError : std::runtime_error {
    lima_status st;
    BuildError(lima_status s, const std::string& m) : std::runtime_error(m), st(s) {}
};
[[noreturn]] void fail(lima_status s, const std::string& m) { throw BuildError(s, m); }

using Row = std::vector<std::string>;

// a value as the next stage reads it: printed with "%f", parsed with strtof
float rt(float v) {
    char b[96];
    std::snprintf(b, sizeof b, "%f", (double)v);
    return std::strtof(b, nullptr);
}
float to_f(const std::string& s) {
    try {
        return std::stof(s);
    } catch (...) {
        fail(LIMA_ERR_ARGUMENT, "not a number: '" + s + "'");
    }
}
int to_i(const std::string& s) {
    try {
        return std::stoi(s);
    } catch (...) {
        fail(LIMA_ERR_ARGUMENT, "not an integer: '" + s + "'");
    }
}

std::vector<std::string> lines_of(const char* path) {
    std::ifstream f(path);
    if (!f) fail(LIMA_ERR_ARGUMENT, std::string("cannot open ") + path);
    std::vector<std::string> out;
    std::string line;
    while (std::getline(f, line)) out.push_back(line);
    return out;
}

// The force-field stage's reader (Filehandling.h:30-99): a line whose first
// non-blank character is ';', '#' or '!' is dropped; fields split on blanks
// and tabs.
std::vector<Row> read_ff_rows(const std::vector<std::string>& lines) {
    std::vector<Row> rows;
    for (const std::string& line : lines) {
        if (line.empty()) continue;
        char first = ' ';
        for (char c : line)
            if (c != ' ' && c != '\t') {
                first = c;
                break;
            }
        if (first == ';' || first == '#' || first == '!') continue;
        Row r;
        std::string cur;
        for (char c : line) {
            if (c == ' ' || c == '\t') {
                if (!cur.empty()) r.push_back(cur);
                cur.clear();
            } else {
                cur += c;
            }
        }
        if (!cur.empty()) r.push_back(cur);
        rows.push_back(r);
    }
    return rows;
}

// The molecule stage's reader (CompoundBuilder.cpp:323-352, 392-418): fields
// split on blanks only; "", "[" and "]" dropped; for the topology a record
// whose first field is ";" is dropped.
Row split_blanks(const std::string& line) {
    Row r;
    std::string cur;
    for (char c : line) {
        if (c == ' ') {
            if (!cur.empty() && cur != "[" && cur != "]") r.push_back(cur);
            cur.clear();
        } else {
            cur += c;
        }
    }
    if (!cur.empty() && cur != "[" && cur != "]") r.push_back(cur);
    return r;
}

// ------------------------------------------------------------ force field --
struct NBType {
    std::string type;
    float mass = -1.f, sigma = -1.f, epsilon = -1.f;
    int local = 0;
};
struct BondT {
    std::string t1, t2;
    int id1 = 0, id2 = 0;
    float b0 = 0.f, kb = 0.f;
};
struct AngleT {
    std::string t1, t2, t3;
    int id1 = 0, id2 = 0, id3 = 0;
    float th0 = 0.f, k = 0.f;
};
struct DihT {
    std::string t1, t2, t3, t4;
    int id1 = 0, id2 = 0, id3 = 0, id4 = 0;
    float phi0 = 0.f, k = 0.f;
    int n = 0;
};

// order two type names character by character; a longer name with an equal
// prefix goes right (Bondtype::sort, ForcefieldTypes.h:364-388)
void sort_pair(std::string& a, std::string& b) {
    size_t p = 0;
    while (a.size() > p && b.size() > p) {
        if (a[p] < b[p]) return;
        if (a[p] > b[p]) {
            std::swap(a, b);
            return;
        }
        p++;
    }
    if (a.size() > b.size()) std::swap(a, b);
}
// FTHelpers::isSorted (ForcefieldTypes.h:42-56): the reference reaches the end
// of the function without a return when one name is a prefix of the other;
// its build treats that path as "not sorted"
bool is_sorted_names(const std::string& l, const std::string& r) {
    size_t p = 0;
    while (l.size() > p && r.size() > p) {
        if (l[p] < r[p]) return true;
        if (l[p] > r[p]) return false;
        p++;
    }
    return false;
}
void sort_dih(DihT& d) {   // Dihedraltype::sort (ForcefieldTypes.h:698-711)
    const bool flip = d.t1 != d.t4 ? !is_sorted_names(d.t1, d.t4) : !is_sorted_names(d.t2, d.t3);
    if (flip) {
        std::swap(d.t1, d.t4);
        std::swap(d.t2, d.t3);
    }
}

// fraction of a shared prefix (FTHelpers::calcLikeness, ForcefieldTypes.h:29-40)
float likeness(const std::string& a, const std::string& b) {
    float l = 0.f;
    const float step = 1.f / (float)std::max(a.size(), b.size());
    for (size_t i = 0; i < std::min(a.size(), b.size()); i++) {
        if (a[i] == b[i]) l += step;
        else break;
    }
    return l;
}

enum PrmState { P_INACTIVE, P_ATOMS, P_BONDS, P_ANGLES, P_DIHEDRALS, P_NONBONDED, P_IMPROPER, P_CMAP };
PrmState prm_state(const std::string& s, PrmState cur) {
    if (s == "ATOMS") return P_ATOMS;
    if (s == "BONDS") return P_BONDS;
    if (s == "ANGLES") return P_ANGLES;
    if (s == "DIHEDRALS") return P_DIHEDRALS;
    if (s == "NONBONDED") return P_NONBONDED;
    if (s == "IMPROPER") return P_IMPROPER;
    if (s == "CMAP") return P_CMAP;
    return cur;
}

struct ForceFieldTables {
    std::vector<NBType> nb;        // merged, WATER first
    std::vector<BondT> bonds;
    std::vector<AngleT> angles;
    std::vector<DihT> dihs;
};

// ForcefieldMerger::mergeForcefields (ForcefieldMerger.h:11-170), then the
// round trip through LIMA_ffnonbonded.txt / LIMA_ffbonded.txt
ForceFieldTables merge_prm(const std::vector<std::string>& prm_paths) {
    ForceFieldTables t;
    std::vector<NBType> nb;
    for (const std::string& path : prm_paths) {
        const std::vector<Row> rows = read_ff_rows(lines_of(path.c_str()));
        PrmState st = P_INACTIVE;
        for (const Row& row : rows) {   // atom types and their non-bonded parameters
            if (row.empty()) continue;
            st = prm_state(row[0], st);
            if (st == P_ATOMS) {
                if (row.size() < 4) continue;
                bool dup = false;
                for (const NBType& a : nb) dup = dup || a.type == row[2];
                if (dup) continue;
                NBType a;
                a.type = row[2];
                a.mass = to_f(row[3]);
                nb.push_back(a);
            } else if (st == P_NONBONDED) {
                if (row.size() < 4) continue;
                for (NBType& a : nb)
                    if (a.type == row[0]) {
                        a.epsilon = std::fabs(to_f(row[2]) * 4184.f);   // kcal -> J
                        a.sigma = to_f(row[3]) * 2.f / 10.f;          // Rmin/2 (A) -> 2 Rmin/2 (nm)
                        break;
                    }
            }
        }
        st = P_INACTIVE;
        for (const Row& row : rows) {
            if (row.empty()) continue;
            st = prm_state(row[0], st);
            if (st != P_BONDS || row.size() < 4) continue;
            BondT b;
            b.t1 = row[0];
            b.t2 = row[1];
            b.b0 = to_f(row[3]) * 0.1f;              // A -> nm
            b.kb = to_f(row[2]) * 4183.f * 100.f;    // kcal/(mol A^2) -> J/(mol nm^2), the reference's constants
            sort_pair(b.t1, b.t2);
            bool dup = false;
            for (const BondT& o : t.bonds) dup = dup || (o.t1 == b.t1 && o.t2 == b.t2);
            if (!dup) t.bonds.push_back(b);
        }
        st = P_INACTIVE;
        for (const Row& row : rows) {
            if (row.empty()) continue;
            st = prm_state(row[0], st);
            if (st != P_ANGLES || row.size() < 5) continue;
            AngleT a;
            a.t1 = row[0];
            a.t2 = row[1];
            a.t3 = row[2];
            a.th0 = to_f(row[4]) * 2 * 3.1415f / 360.f;   // degrees -> rad, the reference's pi
            a.k = to_f(row[3]) * 4183.f;
            sort_pair(a.t1, a.t3);
            bool dup = false;
            for (const AngleT& o : t.angles) dup = dup || (o.t1 == a.t1 && o.t2 == a.t2 && o.t3 == a.t3);
            if (!dup) t.angles.push_back(a);
        }
        st = P_INACTIVE;
        for (const Row& row : rows) {
            if (row.empty()) continue;
            st = prm_state(row[0], st);
            if (st != P_DIHEDRALS || row.size() < 7) continue;
            DihT d;
            d.t1 = row[0];
            d.t2 = row[1];
            d.t3 = row[2];
            d.t4 = row[3];
            d.phi0 = to_f(row[6]) * 2 * 3.1415f / 360.f;
            d.k = to_f(row[4]) * 4183.f;
            d.n = to_i(row[5]);
            sort_dih(d);
            bool dup = false;
            for (const DihT& o : t.dihs) dup = dup || (o.t1 == d.t1 && o.t2 == d.t2 && o.t3 == d.t3 && o.t4 == d.t4);
            if (!dup) t.dihs.push_back(d);
        }
    }
    // the reader of the merged tables puts the single-site water first
    // (NB_Atomtype::parseNonbonded, ForcefieldTypes.h:174-204)
    NBType water;
    water.type = "WATER";
    water.mass = (float)(15.999000 + 2 * 1.008000);
    water.sigma = (float)(0.302905564168 + 2 * 0.040001352445);
    water.epsilon = (0.50208f + 2.f * 0.19246f) * 1000.f;
    t.nb.push_back(water);
    for (NBType a : nb) {
        a.mass = rt(a.mass);
        a.sigma = rt(a.sigma);
        a.epsilon = rt(a.epsilon);
        t.nb.push_back(a);
    }
    for (BondT& b : t.bonds) {
        b.b0 = rt(b.b0);
        b.kb = rt(b.kb);
    }
    for (AngleT& a : t.angles) {
        a.th0 = rt(a.th0);
        a.k = rt(a.k);
    }
    for (DihT& d : t.dihs) {
        d.phi0 = rt(d.phi0);
        d.k = rt(d.k);
        // the reader of LIMA_ffbonded.txt builds each entry through the sorting
        // constructor again (ForcefieldTypes.h:718-735); for names where one is
        // a prefix of the other the flip is unconditional, so it undoes the first
        sort_dih(d);
    }
    return t;
}

// ------------------------------------------------------------- molecule ---
struct AtomRec {   // one conf.gro atom (CompoundBuilder::Record_ATOM)
    int serial;
    std::string name, resname;
    int resid;
    float x, y, z;
};

// CompoundBuilder::parseGRO (CompoundBuilder.cpp:392-440)
std::vector<AtomRec> parse_gro(const std::vector<std::string>& lines) {
    std::vector<AtomRec> out;
    for (const std::string& line : lines) {
        Row w = split_blanks(line);
        if (w.empty()) continue;
        std::string id, name;
        for (char c : w[0]) {
            if (c > 47 && c < 58) id += c;
            else name += c;
        }
        const bool valid = !id.empty() && !name.empty();
        if (w.size() == 5) {   // atom name and serial run together (water past 9,999 residues)
            Row v;
            v.push_back(w[0]);
            if (w[1][0] == 'O') {
                v.push_back("OW");
                v.push_back(w[1].size() > 2 ? w[1].substr(2) : std::string());
            } else {
                v.push_back("HW");
                v.push_back(w[1].size() > 3 ? w[1].substr(3) : std::string());
            }
            for (int i = 2; i < 5; i++) v.push_back(w[i]);
            w = v;
        }
        if (!valid || w.size() != 6) continue;
        AtomRec r;
        r.serial = to_i(w[2]);
        r.name = w[1];
        r.resname = name;
        r.resid = to_i(id);
        r.x = (float)std::strtod(w[3].c_str(), nullptr);
        r.y = (float)std::strtod(w[4].c_str(), nullptr);
        r.z = (float)std::strtod(w[5].c_str(), nullptr);
        out.push_back(r);
    }
    return out;
}

int color_type(char c) {   // ForceFieldMaker::atomTypeToIndex (Forcefield.cuh:51-66)
    switch (c) {
        case 'C': return 1;
        case 'O': return 2;
        case 'N': return 3;
        case 'H': return 4;
        case 'P': return 5;
        case 'S': return 6;
        default: fail(LIMA_ERR_ARGUMENT, std::string("no colour type for atom name starting with '") + c + "'");
    }
}

struct PRef {   // ParticleRef (Bodies.cuh:34-47)
    int global = -1, compound = -1, local = -1, local_bridge = -1;
};

struct Bridge {   // CompoundBridge (Bodies.cuh:503-606), host form
    int left, right;
    std::vector<PRef> parts;
    std::vector<uint8_t> types;
    std::vector<lima_pair_bond> bonds;
    std::vector<lima_angle_bond> angles;
    std::vector<lima_dihedral_bond> dihs;
    int local_of(int global) const {
        for (const PRef& p : parts)
            if (p.global == global) return p.local_bridge;
        return global;   // the reference leaves an id it cannot find unchanged
    }
};

void add_ignore(lima_compound& c, int local, int target_local, int target_compound) {   // LJ_Ignores::addIgnoreTarget
    lima_lj_ignores& ig = c.lj_ignore_list[local];
    for (int i = 0; i < ig.n_ignores; i++)
        if (ig.local_ids[i] == (uint8_t)target_local && ig.compound_ids[i] == (uint8_t)target_compound) return;
    if (ig.n_ignores == LIMA_LJ_IGNORES_MAX) fail(LIMA_ERR_CAPACITY, "more than 32 LJ exclusions for one particle");
    ig.local_ids[ig.n_ignores] = (uint8_t)target_local;
    ig.compound_ids[ig.n_ignores] = (uint8_t)target_compound;
    ig.n_ignores++;
}

lima_float3 f3(float x, float y, float z) { return lima_float3{x, y, z}; }
float len3(lima_float3 a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
lima_float3 sub3(lima_float3 a, lima_float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }

// Compound::calcCOM (Bodies.cuh:362-368): sum of prev_positions * (1/n), in float
lima_float3 com_of(const lima_compound& c) {
    lima_float3 com = f3(0.f, 0.f, 0.f);
    const float w = 1.f / (float)c.n_particles;
    for (int i = 0; i < c.n_particles; i++) {
        com.x += c.prev_positions[i].x * w;
        com.y += c.prev_positions[i].y * w;
        com.z += c.prev_positions[i].z * w;
    }
    return com;
}

void build(lima_topology& T, const char* gro, const char* top, const std::vector<std::string>& prms,
           const lima_topology_options& o) {
    const std::vector<std::string> gro_lines = lines_of(gro), top_lines = lines_of(top);
    // ---- stage 1: force field tables and the conf's atom names -> types
    ForceFieldTables ff = merge_prm(prms);
    std::vector<std::string> names;   // FTHelpers::parseConf: distinct names of 6-field conf rows
    for (const Row& r : read_ff_rows(gro_lines)) {
        if (r.size() != 6) continue;
        bool seen = false;
        for (const std::string& n : names) seen = seen || n == r[1];
        if (!seen) names.push_back(r[1]);
    }
    std::vector<NBType> used;   // NB_Atomtype::filterUnusedTypes (ForcefieldTypes.h:228-258)
    std::vector<std::pair<std::string, std::string>> alias_map;
    used.push_back(ff.nb[0]);
    used[0].local = 0;
    for (const std::string& name : names) {
        std::string alias = name;
        for (;;) {
            const NBType* rec = nullptr;
            for (const NBType& a : ff.nb)
                if (a.type == alias) {
                    rec = &a;
                    break;
                }
            if (rec) {
                bool have = false;
                for (const NBType& u : used) have = have || u.type == alias;
                if (!have) {
                    NBType u = *rec;
                    u.local = (int)used.size();
                    used.push_back(u);
                }
                if (name != alias) {
                    bool mapped = false;
                    for (auto& m : alias_map) mapped = mapped || m.first == name;
                    if (!mapped) alias_map.emplace_back(name, alias);
                }
                break;
            }
            if (alias.size() > 1) alias.pop_back();
            else fail(LIMA_ERR_ARGUMENT, "atom name '" + name + "' matches no non-bonded type");
        }
    }
    if ((int)used.size() > LIMA_MAX_ATOM_TYPES) fail(LIMA_ERR_CAPACITY, "more than 32 atom types");
    T.n_types = (int)used.size();
    for (int i = 0; i < T.n_types; i++) {   // Forcefield.cu:81-98, 202-210 (second round trip, g/mol -> kg/mol)
        lima_particle_parameters& p = T.ff.particle_parameters[i];
        p.mass = (float)(rt(used[i].mass) * 1e-3);
        p.sigma = rt(used[i].sigma);
        p.epsilon = rt(used[i].epsilon);
    }
    auto map_right = [&](const std::string& q) {
        for (auto& m : alias_map)
            if (m.first == q) return m.second;
        return q;
    };

    // ---- topology atoms (Atom::parseTopolAtoms / assignAtomtypeIDs, ForcefieldTypes.h:288-340)
    const std::vector<Row> trows = read_ff_rows(top_lines);
    struct TopAtom {
        int id;
        std::string type_bond, name;
        int type_id = -1;
    };
    std::vector<TopAtom> atoms;
    {
        int st = 0;   // 0 inactive, 1 atoms, 2 finished
        for (const Row& r : trows) {
            if (r.size() == 3) {
                if (r[1] == "atoms") st = 1;
                else if (r[1] == "bonds") st = 2;
                continue;
            }
            if (st == 1) {
                if (r.size() < 5) fail(LIMA_ERR_ARGUMENT, "short [ atoms ] row in the topology");
                atoms.push_back(TopAtom{to_i(r[0]), r[1], r[4], -1});
            }
            if (st == 2) break;
        }
    }
    for (TopAtom& a : atoms) {
        const std::string alias = map_right(a.name);
        for (const NBType& u : used)
            if (u.type == alias) a.type_id = u.local;
        if (a.type_id < 0) fail(LIMA_ERR_ARGUMENT, "topology atom '" + a.name + "' has no non-bonded type");
    }
    std::vector<int> type_of_serial;
    for (const TopAtom& a : atoms) {
        if (a.id < 0) fail(LIMA_ERR_ARGUMENT, "negative atom id in the topology");
        if ((size_t)a.id >= type_of_serial.size()) type_of_serial.resize(a.id + 1, -1);
        type_of_serial[a.id] = a.type_id;
    }
    auto atom_at = [&](int id) -> const TopAtom& {
        if (id < 1 || id > (int)atoms.size()) fail(LIMA_ERR_ARGUMENT, "topology term refers to atom " + std::to_string(id));
        return atoms[id - 1];
    };

    // ---- topology terms with force-field parameters (ForcefieldTypes.h:400-520, 580-640, 740-835)
    enum { F_INACTIVE, F_BONDS, F_ANGLES, F_DIHEDRALS, F_PAIRS };
    auto fstate = [](const std::string& s, int cur) {
        if (s == "ff_bondtypes" || s == "bonds") return (int)F_BONDS;
        if (s == "ff_angletypes" || s == "angles") return (int)F_ANGLES;
        if (s == "ff_dihedraltypes" || s == "dihedrals") return (int)F_DIHEDRALS;
        if (s == "pairs") return (int)F_PAIRS;
        return cur;
    };
    std::vector<BondT> tbonds;
    std::vector<AngleT> tangles;
    std::vector<DihT> tdihs;
    {
        int st = F_INACTIVE;
        for (const Row& r : trows) {
            if (r.size() == 3 && r[0][0] == '[') {
                st = fstate(r[1], st);
                continue;
            }
            if (st == F_BONDS) {
                BondT b;
                b.id1 = to_i(r.at(0));
                b.id2 = to_i(r.at(1));
                tbonds.push_back(b);
            }
        }
        st = F_INACTIVE;
        for (const Row& r : trows) {
            if (r.size() == 3 && r[0][0] == '[') {
                st = fstate(r[1], st);
                continue;
            }
            if (st == F_ANGLES) {
                AngleT a;
                a.id1 = to_i(r.at(0));
                a.id2 = to_i(r.at(1));
                a.id3 = to_i(r.at(2));
                tangles.push_back(a);
            }
            if (st == F_DIHEDRALS) break;
        }
        st = F_INACTIVE;
        bool entered = false;
        for (const Row& r : trows) {
            if (r.size() == 3 && r[0][0] == '[') {
                st = fstate(r[1], st);
                if (entered) break;
                continue;
            }
            if (st == F_DIHEDRALS) {
                if (r.size() != 5) continue;
                DihT d;
                d.id1 = to_i(r[0]);
                d.id2 = to_i(r[1]);
                d.id3 = to_i(r[2]);
                d.id4 = to_i(r[3]);
                tdihs.push_back(d);
                entered = true;
            }
        }
    }
    for (BondT& b : tbonds) {
        b.t1 = atom_at(b.id1).type_bond;
        b.t2 = atom_at(b.id2).type_bond;
        sort_pair(b.t1, b.t2);
        float best = 0.f;
        const BondT* m = nullptr;
        for (const BondT& f : ff.bonds) {
            const float l = likeness(b.t1, f.t1) * likeness(b.t2, f.t2);
            if (l > best) {
                best = l;
                m = &f;
            }
        }
        if (!(best > 0.01f) || !m) fail(LIMA_ERR_ARGUMENT, "no bond parameters for types " + b.t1 + " " + b.t2);
        b.b0 = m->b0;
        b.kb = m->kb;
    }
    for (AngleT& a : tangles) {
        a.t1 = atom_at(a.id1).type_bond;
        a.t2 = atom_at(a.id2).type_bond;
        a.t3 = atom_at(a.id3).type_bond;
        sort_pair(a.t1, a.t3);
        float best = 0.f;
        const AngleT* m = nullptr;
        for (const AngleT& f : ff.angles) {
            const float l = likeness(a.t1, f.t1) * likeness(a.t2, f.t2) * likeness(a.t3, f.t3);
            if (l > best) {
                best = l;
                m = &f;
            }
            if (l == 1.f) break;
        }
        if (!(best > 0.01f) || !m) fail(LIMA_ERR_ARGUMENT, "no angle parameters for types " + a.t1 + " " + a.t2 + " " + a.t3);
        a.th0 = m->th0;
        a.k = m->k;
    }
    for (DihT& d : tdihs) {
        d.t1 = atom_at(d.id1).type_bond;
        d.t2 = atom_at(d.id2).type_bond;
        d.t3 = atom_at(d.id3).type_bond;
        d.t4 = atom_at(d.id4).type_bond;
        sort_dih(d);
        float best = 0.f;
        const DihT* m = nullptr;
        for (const DihT& f : ff.dihs) {
            const float l = likeness(d.t1, f.t1) * likeness(d.t2, f.t2) * likeness(d.t3, f.t3) * likeness(d.t4, f.t4);
            if (l > best) {
                best = l;
                m = &f;
            }
            if (l == 1.f) break;
        }
        if (!(best > 0.001f) || !m) fail(LIMA_ERR_ARGUMENT, "no dihedral parameters for types " + d.t1 + " " + d.t2);
        d.phi0 = m->phi0;
        d.k = m->k;
        d.n = m->n;
    }
    // the round trip through LIMA_ffbonded_filtered.txt into ForceFieldMaker (Forcefield.cu:116-200);
    // dihedral force constants are taken as |k_phi|
    for (BondT& b : tbonds) {
        b.b0 = rt(b.b0);
        b.kb = rt(b.kb);
    }
    for (AngleT& a : tangles) {
        a.th0 = rt(a.th0);
        a.k = rt(a.k);
    }
    for (DihT& d : tdihs) {
        d.phi0 = rt(d.phi0);
        d.k = std::fabs(rt(d.k));
    }

    // ---- stage 3: molecule (CompoundBuilder::loadParticles / loadTopology)
    const std::vector<AtomRec> recs = parse_gro(gro_lines);
    std::vector<PRef> ref_of;   // by serial
    auto ref_at = [&](int serial) -> PRef {
        if (serial < 0 || (size_t)serial >= ref_of.size()) return PRef{};
        return ref_of[serial];
    };
    std::vector<lima_compound>& comps = T.comps;
    std::vector<Bridge> bridges;
    int n_atoms_total = 0;
    {
        int cur_res = -1;
        lima_compound* cur = nullptr;
        for (const AtomRec& r : recs) {
            if (r.resid < o.min_residue_id) continue;
            if (r.resid > o.max_residue_id) break;
            if (o.ignore_hydrogens && r.name[0] == 'H') continue;
            if (r.resname == "SOL") continue;
            if (r.resid != cur_res) {
                // Compound::hasRoomForRes: room for a residue of up to 32 atoms
                if (cur == nullptr || (int)cur->n_particles + 32 > LIMA_MAX_COMPOUND_PARTICLES) {
                    if (cur != nullptr) {
                        const int l = (int)comps.size() - 1;
                        if ((int)bridges.size() == 64) fail(LIMA_ERR_CAPACITY, "more than 64 compound bridges");
                        bridges.push_back(Bridge{l, l + 1, {}, {}, {}, {}, {}});
                    }
                    if ((int)comps.size() == LIMA_MAX_COMPOUNDS) fail(LIMA_ERR_CAPACITY, "more than 255 compounds");
                    comps.emplace_back();
                    std::memset(&comps.back(), 0, sizeof(lima_compound));
                    comps.back().key_particle_index = 404;
                    cur = &comps.back();
                }
                cur_res = r.resid;
            }
            if (cur->n_particles == LIMA_MAX_COMPOUND_PARTICLES) fail(LIMA_ERR_CAPACITY, "compound overflow");
            if (r.serial < 1 || (size_t)r.serial >= type_of_serial.size() || type_of_serial[r.serial] < 0)
                fail(LIMA_ERR_ARGUMENT, "conf atom " + std::to_string(r.serial) + " is not in the topology");
            if ((size_t)r.serial >= ref_of.size()) ref_of.resize(r.serial + 1);
            ref_of[r.serial] = PRef{r.serial, (int)comps.size() - 1, cur->n_particles, -1};
            const int k = cur->n_particles;
            cur->atom_types[k] = (uint8_t)type_of_serial[r.serial];
            cur->prev_positions[k] = f3(r.x, r.y, r.z);
            cur->atom_color_types[k] = (uint8_t)color_type(r.name[0]);
            cur->particle_global_ids[k] = (uint32_t)r.serial;
            cur->n_particles++;
            n_atoms_total++;
        }
    }
    if (comps.empty()) fail(LIMA_ERR_ARGUMENT, "no atoms selected from the conf");
    // terms in topology order; parameters from the tables above by exact id order
    auto bond_params = [&](int a, int b) -> const BondT& {
        for (const BondT& x : tbonds)
            if (x.id1 == a && x.id2 == b) return x;
        fail(LIMA_ERR_ARGUMENT, "bond " + std::to_string(a) + "-" + std::to_string(b) + " has no parameters");
    };
    auto angle_params = [&](int a, int b, int c) -> const AngleT& {
        for (const AngleT& x : tangles)
            if (x.id1 == a && x.id2 == b && x.id3 == c) return x;
        fail(LIMA_ERR_ARGUMENT, "angle without parameters");
    };
    auto dih_params = [&](int a, int b, int c, int d) -> const DihT& {
        for (const DihT& x : tdihs)
            if (x.id1 == a && x.id2 == b && x.id3 == c && x.id4 == d) return x;
        fail(LIMA_ERR_ARGUMENT, "dihedral without parameters");
    };
    auto bridge_of = [&](const PRef* m, int n) -> Bridge* {
        int c0 = -1, c1 = -1;   // GenericBond: first compound seen, then any other
        for (int i = 0; i < n; i++) {
            if (c0 == -1) c0 = m[i].compound;
            else if (c0 != m[i].compound) c1 = m[i].compound;
        }
        if (c1 == -1) return nullptr;
        if (c0 > c1) std::swap(c0, c1);
        for (Bridge& b : bridges)
            if (b.left == c0 && b.right == c1) return &b;
        fail(LIMA_ERR_ARGUMENT, "a term spans compounds " + std::to_string(c0) + " and " + std::to_string(c1) +
                                     " that are not consecutive");
    };
    auto add_bridge_particles = [&](Bridge& b, PRef* m, int n) {
        for (int i = 0; i < n; i++) {
            bool stored = false;
            for (const PRef& p : b.parts) stored = stored || p.global == m[i].global;
            if (stored) continue;
            if ((int)b.parts.size() == LIMA_MAX_PARTICLES_IN_BRIDGE) fail(LIMA_ERR_CAPACITY, "bridge overflow");
            PRef p = m[i];
            p.local_bridge = (int)b.parts.size();
            b.types.push_back(comps[p.compound].atom_types[p.local]);
            b.parts.push_back(p);
        }
    };
    auto exclude = [&](const PRef* m, int n) {   // CompoundBuilder::distributeLJIgnores
        for (int s = 0; s < n; s++)
            for (int t = 0; t < n; t++)
                if (s != t) add_ignore(comps[m[s].compound], m[s].local, m[t].local, m[t].compound);
    };
    {
        enum { M_INACTIVE, M_BOND, M_ANGLE, M_DIHEDRAL };
        int mode = M_INACTIVE, dih_sections = 0;
        for (const std::string& line : top_lines) {
            const Row r = split_blanks(line);
            if (!r.empty() && r[0] == ";") continue;
            if (r.empty()) {
                mode = M_INACTIVE;
                continue;
            }
            if (mode == M_INACTIVE) {
                mode = r[0] == "bonds" ? M_BOND : r[0] == "angles" ? M_ANGLE : r[0] == "dihedrals" ? M_DIHEDRAL : M_INACTIVE;
                if (mode == M_DIHEDRAL) dih_sections++;
                continue;
            }
            if (mode == M_DIHEDRAL && dih_sections > 1) continue;   // the second section holds the impropers
            const int n = mode == M_BOND ? 2 : mode == M_ANGLE ? 3 : 4;
            if ((int)r.size() < n) fail(LIMA_ERR_ARGUMENT, "short term row in the topology");
            PRef m[4];
            int id[4];
            bool all = true;
            for (int i = 0; i < n; i++) {
                id[i] = to_i(r[i]);
                m[i] = ref_at(id[i]);
                all = all && m[i].local != -1;
            }
            if (!all) continue;   // a term with a left-out atom (hydrogens) is dropped
            Bridge* br = bridge_of(m, n);
            if (mode == M_BOND) {
                const BondT& p = bond_params(id[0], id[1]);
                exclude(m, 2);
                if (!br) {
                    lima_compound& c = comps[m[0].compound];
                    if (c.n_singlebonds == LIMA_MAX_PAIRBONDS) fail(LIMA_ERR_CAPACITY, "too many bonds in a compound");
                    c.singlebonds[c.n_singlebonds++] = lima_pair_bond{p.b0, p.kb, {(uint32_t)m[0].local, (uint32_t)m[1].local}};
                } else {
                    add_bridge_particles(*br, m, 2);
                    if ((int)br->bonds.size() == LIMA_MAX_SINGLEBONDS_IN_BRIDGE) fail(LIMA_ERR_CAPACITY, "bridge bonds");
                    br->bonds.push_back(lima_pair_bond{p.b0, p.kb,
                                                       {(uint32_t)br->local_of(id[0]), (uint32_t)br->local_of(id[1])}});
                }
            } else if (mode == M_ANGLE) {
                const AngleT& p = angle_params(id[0], id[1], id[2]);
                exclude(m, 3);
                if (!br) {
                    lima_compound& c = comps[m[0].compound];
                    if (c.n_anglebonds == LIMA_MAX_ANGLEBONDS) fail(LIMA_ERR_CAPACITY, "too many angles in a compound");
                    c.anglebonds[c.n_anglebonds++] =
                        lima_angle_bond{p.th0, p.k, {(uint32_t)m[0].local, (uint32_t)m[1].local, (uint32_t)m[2].local}};
                } else {
                    add_bridge_particles(*br, m, 3);
                    if ((int)br->angles.size() == LIMA_MAX_ANGLEBONDS_IN_BRIDGE) fail(LIMA_ERR_CAPACITY, "bridge angles");
                    br->angles.push_back(lima_angle_bond{
                        p.th0, p.k,
                        {(uint32_t)br->local_of(id[0]), (uint32_t)br->local_of(id[1]), (uint32_t)br->local_of(id[2])}});
                }
            } else {
                const DihT& p = dih_params(id[0], id[1], id[2], id[3]);
                exclude(m, 4);
                lima_dihedral_bond db{};
                db.phi_0 = p.phi0;
                db.k_phi = p.k;
                db.n = (uint8_t)p.n;
                if (!br) {
                    lima_compound& c = comps[m[0].compound];
                    if (c.n_dihedrals == LIMA_MAX_DIHEDRALS) fail(LIMA_ERR_CAPACITY, "too many dihedrals in a compound");
                    for (int i = 0; i < 4; i++) db.atom_indexes[i] = (uint32_t)m[i].local;
                    c.dihedrals[c.n_dihedrals++] = db;
                } else {
                    add_bridge_particles(*br, m, 4);
                    if ((int)br->dihs.size() == LIMA_MAX_DIHEDRALBONDS_IN_BRIDGE) fail(LIMA_ERR_CAPACITY, "bridge dihedrals");
                    for (int i = 0; i < 4; i++) db.atom_indexes[i] = (uint32_t)br->local_of(id[i]);
                    br->dihs.push_back(db);
                }
            }
        }
    }
    // Compound::calcParticleSphere (Bodies.cuh:407-420), on the conf's own coordinates
    for (lima_compound& c : comps) {
        const lima_float3 com = com_of(c);
        float furthest = (float)LONG_MIN, closest = (float)LONG_MAX;
        int closest_index = 0;
        for (int i = 0; i < c.n_particles; i++) {
            const float d = len3(sub3(c.prev_positions[i], com));
            closest_index = d < closest ? i : closest_index;
            closest = std::min(closest, d);
            furthest = std::max(furthest, d);
        }
        c.key_particle_index = closest_index;
        c.confining_particle_sphere = furthest;
    }
    // ---- box (BoxBuilder::addSingleMolecule / integrateCompound): centre of the compound
    // centres at the box centre; previous positions equal to the positions (no velocity)
    lima_float3 mcom = f3(0.f, 0.f, 0.f);
    {
        const float w = 1.f / (float)comps.size();
        for (const lima_compound& c : comps) {
            const lima_float3 cc = com_of(c);
            mcom.x += cc.x * w;
            mcom.y += cc.y * w;
            mcom.z += cc.z * w;
        }
    }
    const float half = o.box_len / 2.f;
    const lima_float3 off = f3(half - mcom.x, half - mcom.y, half - mcom.z);
    T.states.resize(comps.size());
    for (size_t ci = 0; ci < comps.size(); ci++) {
        lima_compound& c = comps[ci];
        for (int i = 0; i < c.n_particles; i++) {
            c.prev_positions[i].x += off.x;
            c.prev_positions[i].y += off.y;
            c.prev_positions[i].z += off.z;
        }
        c.center_of_mass = com_of(c);
        lima_compound_state& s = T.states[ci];
        std::memset(&s, 0, sizeof s);
        for (int i = 0; i < c.n_particles; i++) s.positions[i] = c.prev_positions[i];
        s.n_particles = c.n_particles;
    }
    // bridges in the reference's compact form
    for (const Bridge& b : bridges) {
        lima_compound_bridge_compact bc{};
        std::memset(&bc, 0, sizeof bc);
        bc.n_particles = (int32_t)b.parts.size();
        for (size_t i = 0; i < b.parts.size(); i++) {
            bc.particle_refs[i] = lima_particle_ref_compact{b.parts[i].compound, b.parts[i].local};
            bc.atom_types[i] = b.types[i];
        }
        bc.n_singlebonds = (uint16_t)b.bonds.size();
        for (size_t i = 0; i < b.bonds.size(); i++) bc.singlebonds[i] = b.bonds[i];
        bc.n_anglebonds = (uint16_t)b.angles.size();
        for (size_t i = 0; i < b.angles.size(); i++) bc.anglebonds[i] = b.angles[i];
        bc.n_dihedrals = (uint16_t)b.dihs.size();
        for (size_t i = 0; i < b.dihs.size(); i++) bc.dihedrals[i] = b.dihs[i];
        T.bridges.push_back(bc);
    }
    // ---- solvents (CompoundBuilder::getSolventPositions + BoxBuilder::solvateBox / spaceAvailable)
    if (o.solvate) {
        const double v_rms = std::sqrt(3.0 * 8.3144 * o.temperature / (double)(18.01528f * 1e-3));
        uint64_t s = o.seed ? o.seed : 0x9E3779B97F4A7C15ull;
        auto next = [&]() {   // splitmix64
            uint64_t z = (s += 0x9E3779B97F4A7C15ull);
            z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
            z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
            return (double)((z ^ (z >> 31)) >> 11) * (1.0 / 9007199254740992.0);
        };
        for (const AtomRec& r : recs) {
            if (r.resname != "SOL" || r.name[0] != 'O') continue;
            if ((int)T.sols.size() == 0xFFFF) fail(LIMA_ERR_CAPACITY, "more than 65,535 solvents");
            const lima_float3 p = f3(r.x + off.x, r.y + off.y, r.z + off.z);
            bool room = true;
            for (const lima_compound& c : comps) {
                float md = 999999.f;
                for (int i = 0; i < c.n_particles && room; i++) md = std::min(md, len3(sub3(c.prev_positions[i], p)));
                if (md < 0.2f) room = false;
                if (!room) break;
            }
            for (size_t q = 0; q < T.sols.size() && room; q++)
                if (len3(sub3(T.sols[q].pos, p)) < 0.25f) room = false;
            if (!room) continue;
            // a direction uniform on the sphere, at the reference's speed
            const double u = 2.0 * next() - 1.0, phi = 2.0 * M_PI * next(), st = std::sqrt(std::max(0.0, 1.0 - u * u));
            const double vx = v_rms * st * std::cos(phi), vy = v_rms * st * std::sin(phi), vz = v_rms * u;
            lima_solvent sol;
            sol.pos = p;
            sol.pos_tsub1 = f3(p.x - (float)(vx * o.dt), p.y - (float)(vy * o.dt), p.z - (float)(vz * o.dt));
            T.sols.push_back(sol);
        }
    }
    (void)n_atoms_total;
}

}  // namespace

extern "C" {

void lima_topology_default_options(lima_topology_options* o) {
    if (!o) return;
    o->box_len = 7.f;            // Constants.cuh:35
    o->min_residue_id = 0;       // Environment.cpp:21-23
    o->max_residue_id = 200;
    o->ignore_hydrogens = 1;
    o->solvate = 1;
    o->dt = 1e-7;                // Simulation.cuh:152
    o->temperature = 313.0;      // BoxBuilder.cuh:67
    o->seed = 2024;
}

lima_status lima_topology_build(const char* gro_path, const char* top_path, const char* const* prm_paths, int n_prm,
                                const lima_topology_options* options, lima_topology** out) {
    if (!out) return LIMA_ERR_ARGUMENT;
    *out = nullptr;
    lima_topology* t = nullptr;
    try {
        t = new lima_topology();
    } catch (...) {
        return LIMA_ERR_ARGUMENT;
    }
    *out = t;
    try {
        if (!gro_path || !top_path || n_prm < 1 || !prm_paths) fail(LIMA_ERR_ARGUMENT, "need conf, topology and >= 1 parameter file");
        lima_topology_options o;
        lima_topology_default_options(&o);
        if (options) o = *options;
        if (!(o.box_len > 0.f) || !(o.dt > 0.0)) fail(LIMA_ERR_ARGUMENT, "box_len and dt must be positive");
        std::vector<std::string> prms;
        for (int i = 0; i < n_prm; i++) {
            if (!prm_paths[i]) fail(LIMA_ERR_ARGUMENT, "null parameter file path");
            prms.emplace_back(prm_paths[i]);
        }
        build(*t, gro_path, top_path, prms, o);
        return LIMA_OK;
    } catch (const BuildError& e) {
        t->err = e.what();
        return e.st;
    } catch (const std::exception& e) {
        t->err = e.what();
        return LIMA_ERR_ARGUMENT;
    }
}

const char* lima_topology_error(const lima_topology* t) { return t ? t->err.c_str() : "null topology"; }

lima_status lima_topology_sizes(const lima_topology* t, int* n_compounds, int* n_bridges, uint32_t* n_solvents,
                                int* n_atom_types) {
    if (!t || !t->err.empty()) return LIMA_ERR_STATE;
    if (n_compounds) *n_compounds = (int)t->comps.size();
    if (n_bridges) *n_bridges = (int)t->bridges.size();
    if (n_solvents) *n_solvents = (uint32_t)t->sols.size();
    if (n_atom_types) *n_atom_types = t->n_types;
    return LIMA_OK;
}

lima_status lima_topology_export(const lima_topology* t, lima_forcefield* ff, lima_compound* compounds,
                                 lima_compound_state* states, lima_compound_bridge_compact* bridges,
                                 lima_solvent* solvents) {
    if (!t || !t->err.empty()) return LIMA_ERR_STATE;
    if (ff) *ff = t->ff;
    if (compounds && !t->comps.empty()) std::memcpy(compounds, t->comps.data(), sizeof(lima_compound) * t->comps.size());
    if (states && !t->states.empty())
        std::memcpy(states, t->states.data(), sizeof(lima_compound_state) * t->states.size());
    if (bridges && !t->bridges.empty())
        std::memcpy(bridges, t->bridges.data(), sizeof(lima_compound_bridge_compact) * t->bridges.size());
    if (solvents && !t->sols.empty()) std::memcpy(solvents, t->sols.data(), sizeof(lima_solvent) * t->sols.size());
    return LIMA_OK;
}

void lima_topology_destroy(lima_topology* t) { delete t; }

}  // extern "C"
