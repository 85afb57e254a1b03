// BoundaryConditions.txt parser of the C ABI (acp_parse_case_file).
//
// Keyword rules of Control::readValue / readString (Control.cpp:135-204): the
// file is scanned line by line, the first whitespace-separated token must
// equal the keyword exactly (so "//" and "#" lines never match), the value is
// the next token read by stream extraction (a number stops at ';' or a
// comment), and a missing mandatory keyword is an error naming the keyword
// (the reference prints it and exits, Control.cpp:163-164).  The node counts
// follow Control.cpp:43-45: ceil(size / spacing + 1e-8).  Keywords added by
// this engine are optional and default to the reference's behaviour.
#include "../../include/acp.h"

#include <cmath>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <string>

namespace {

bool findLine(const std::string& path, const std::string& key, std::string& rest, bool& fileOk) {
    std::ifstream in(path);
    fileOk = (bool)in;
    if (!in) return false;
    std::string line;
    while (std::getline(in, line)) {
        std::istringstream s(line);
        std::string op;
        if (!(s >> op)) continue;
        if (op == key) {
            std::getline(s, rest);
            return true;
        }
    }
    return false;
}

struct Parser {
    std::string path;
    std::string err;
    bool ok = true;

    bool value(const char* key, double& out, bool required = true) {
        std::string rest;
        bool fileOk;
        if (!findLine(path, key, rest, fileOk)) {
            if (!fileOk) { err = "Error reading boundary conditions file " + path; ok = false; }
            else if (required) { err = std::string("No Value for keyword \"") + key + "\" found in " + path; ok = false; }
            return false;
        }
        std::istringstream s(rest);
        double v = 0.;
        s >> v;  // like the reference: a non-number reads as 0
        out = v;
        return true;
    }
    bool word(const char* key, std::string& out, bool required = true) {
        std::string rest;
        bool fileOk;
        if (!findLine(path, key, rest, fileOk)) {
            if (!fileOk) { err = "Error reading boundary conditions file " + path; ok = false; }
            else if (required) { err = std::string("No Value for keyword \"") + key + "\" found in " + path; ok = false; }
            return false;
        }
        std::istringstream s(rest);
        s >> out;
        return true;
    }
    bool ints(const char* key, int* v, int n) {
        std::string rest;
        bool fileOk;
        if (!findLine(path, key, rest, fileOk)) return false;
        std::istringstream s(rest);
        for (int i = 0; i < n; ++i) s >> v[i];
        return true;
    }
    bool doubles(const char* key, double* v, int n) {
        std::string rest;
        bool fileOk;
        if (!findLine(path, key, rest, fileOk)) return false;
        std::istringstream s(rest);
        for (int i = 0; i < n; ++i) s >> v[i];
        return true;
    }
};

int lookup(const std::string& w, const char* const* names, int n) {
    for (int i = 0; i < n; ++i)
        if (w == names[i]) return i;
    return -1;
}

}  // namespace

extern "C" int acp_parse_case_file(const char* path, acp_case_desc* d, char* errbuf, size_t errlen) {
    if (!path || !d) return ACP_ERR_INVALID;
    acp_default_case(d);
    Parser p;
    p.path = path;
    double v;
    std::string w;
    auto bad = [&](const std::string& m) {
        if (errbuf && errlen) std::snprintf(errbuf, errlen, "%s", m.c_str());
        return ACP_ERR_INVALID;
    };
    // mandatory keywords, in the order of Control::Control (Control.cpp:8-37)
    const char* mandatoryNum[] = {"Max-Time-Step", "WriteInterval", "Density", "Threads", "KinematicViscosity",
                                  "SpeedOfSound", "Order-Of-Equilibrium", "K1-Relaxation", "K2-Relaxation",
                                  "Hybrid-Parameter", "Domain-Size-X", "Domain-Size-Y", "Domain-Size-Z", "Spacing",
                                  "RefinementLayerYZ", "RefinementLayerX", "MaxLevel", "MACH-Number", "Overlap"};
    for (const char* k : mandatoryNum)
        if (!p.value(k, v)) return bad(p.err);
    const char* mandatoryWord[] = {"Save-as", "Collision-Model", "Cubic-Mach-Correction", "Coarse-to-Fine",
                                   "Fine-to-Coarse", "Hanging-Node-Reconstruction", "Scaling-Style", "F2C-Filter",
                                   "Coupling-Approach", "Non-Reflecting", "Transverse"};
    for (const char* k : mandatoryWord)
        if (!p.word(k, w)) return bad(p.err);

    p.value("Density", d->density);
    p.value("KinematicViscosity", d->kinematic_viscosity);
    p.value("SpeedOfSound", d->speed_of_sound);
    p.value("MACH-Number", d->mach);
    p.value("Order-Of-Equilibrium", v); d->eq_order = (int)v;
    p.value("Hybrid-Parameter", d->hybrid_sigma);
    p.value("K1-Relaxation", d->k1);
    p.value("Domain-Size-X", d->domain_size[0]);
    p.value("Domain-Size-Y", d->domain_size[1]);
    p.value("Domain-Size-Z", d->domain_size[2]);
    p.value("Spacing", d->spacing);
    p.value("MaxLevel", v); d->max_level = (int)v;
    p.value("RefinementLayerYZ", v); d->ref_layer_yz = (int)v;
    p.value("RefinementLayerX", v); d->ref_layer_x = (int)v;
    p.value("Overlap", v); d->overlap = (int)v;

    static const char* ops[] = {"SRT", "MRT-GS", "MRT-RM", "RR", "HRR"};
    p.word("Collision-Model", w);
    if ((d->op = lookup(w, ops, 5)) < 0) return bad("unknown Collision-Model " + w);
    p.word("Cubic-Mach-Correction", w); d->cubic_mach = w == "yes";
    p.word("Transverse", w); d->transverse = w == "yes";
    static const char* coup[] = {"STD", "DC1", "DC2"};
    p.word("Coupling-Approach", w);
    if ((d->coupling = lookup(w, coup, 3)) < 0) return bad("unknown Coupling-Approach " + w);
    static const char* filt[] = {"NOFI", "LAG", "TOU"};
    p.word("F2C-Filter", w);
    if ((d->f2c_filter = lookup(w, filt, 3)) < 0) return bad("unknown F2C-Filter " + w);
    static const char* sty[] = {"SRTSTYLE", "MRTSTYLE"};
    p.word("Scaling-Style", w);
    if ((d->scaling_style = lookup(w, sty, 2)) < 0) return bad("unknown Scaling-Style " + w);
    static const char* c2f[] = {"Mf", "MfP", "fAll"};
    p.word("Coarse-to-Fine", w);
    if ((d->c2f_replace = lookup(w, c2f, 3)) < 0) return bad("unknown Coarse-to-Fine " + w);
    static const char* f2c[] = {"Mc", "McP", "cAll"};
    p.word("Fine-to-Coarse", w);
    if ((d->f2c_replace = lookup(w, f2c, 3)) < 0) return bad("unknown Fine-to-Coarse " + w);

    const double eps = 1e-8;  // Control.cpp:40-45
    d->nx = (int)std::ceil(d->domain_size[0] / d->spacing + eps);
    d->ny = (int)std::ceil(d->domain_size[1] / d->spacing + eps);
    d->nz = (int)std::ceil(d->domain_size[2] / d->spacing + eps);

    // optional keywords of this engine
    const char* per[] = {"Periodic-X", "Periodic-Y", "Periodic-Z"};
    for (int a = 0; a < 3; ++a)
        if (p.word(per[a], w, false)) d->bc[a] = w == "yes" ? ACP_BC_PERIODIC : ACP_BC_LODI;
    if (p.word("MRT-Write-Back", w, false)) d->mrt_writeback = w == "yes";
    if (p.word("Storage", w, false)) {
        static const char* st[] = {"FP64", "FP32-DEV", "FP16-DEV"};
        if ((d->storage = lookup(w, st, 3)) < 0) return bad("unknown Storage " + w);
    }
    if (p.word("Refinement-Layout", w, false) && w == "BOX") {
        d->layout = ACP_LAYOUT_BOX;
        if (!p.ints("Refinement-Box-Lo", d->box_lo, 3) || !p.ints("Refinement-Box-Hi", d->box_hi, 3))
            return bad("Refinement-Layout BOX needs Refinement-Box-Lo and Refinement-Box-Hi");
    }
    if (p.value("Pulse-Amplitude", v, false)) {
        d->ic = ACP_IC_GAUSSIAN;
        d->ic_eps = v;
        if (!p.value("Pulse-Halfwidth", d->ic_b, false)) return bad("Pulse-Amplitude needs Pulse-Halfwidth");
        if (!p.doubles("Pulse-Center", d->ic_center, 3)) return bad("Pulse-Amplitude needs Pulse-Center");
        if (p.value("Pulse-Dimensions", v, false)) d->ic_dims = (int)v;
    }
    return ACP_OK;
}
