/*
 * LOQUAT-B200 input/output formats (reference src/loquat_io.cu:69-370).
 *
 *  <project>.xml  <parameters> with typed children <key type="int|float">v</key>
 *                 (reference src/loquat_io.cu:95-119); the key set, the
 *                 model-dependent keys and the np = npb + npm check follow
 *                 src/loquat_io.cu:121-197.
 *  <project>.dat  one particle per line, 22 columns: pospres.xyzw,
 *                 velrhop.xyzw, idep.xy, str (6), stn (6)
 *                 (reference src/loquat_io.cu:226, written in the same order
 *                 at :362).  idep.z and idep.w are not stored and read as 0.
 *
 * Differences from the reference writer, all so that an output pair reads
 * back as an input pair: the DP shear modulus is written under the key the
 * reader expects (elastic-G; the reference writes poisson-G,
 * src/loquat_io.cu:272), and numbers are written with the shortest
 * representation that reads back to the same float instead of 6 digits.
 * Errors return a status with a message; nothing exits the process.
 */
#include <algorithm>
#include <cerrno>
#include <charconv>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "lq_internal.cuh"

namespace {

using lqb::set_error;

struct XmlValue {
    bool is_int;
    int i;
    float f;
};

bool read_file(const char* path, std::string& out)
{
    FILE* fp = fopen(path, "rb");
    if (!fp) return false;
    char buf[1 << 16];
    size_t n;
    out.clear();
    while ((n = fread(buf, 1, sizeof(buf), fp)) > 0) out.append(buf, n);
    fclose(fp);
    return true;
}

inline bool is_space(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r'; }

/* Parses the children of <parameters>.  Returns LQ_OK or LQ_ERR_IO. */
int parse_parameters_xml(const std::string& s, std::map<std::string, XmlValue>& kv)
{
    size_t p = s.find("<parameters");
    if (p == std::string::npos) return set_error(LQ_ERR_IO, "XML: no <parameters> element");
    p = s.find('>', p);
    if (p == std::string::npos) return set_error(LQ_ERR_IO, "XML: unterminated <parameters> tag");
    ++p;
    for (;;) {
        while (p < s.size() && is_space(s[p])) ++p;
        if (p >= s.size()) return set_error(LQ_ERR_IO, "XML: missing </parameters>");
        if (s.compare(p, 4, "<!--") == 0) {
            size_t e = s.find("-->", p);
            if (e == std::string::npos) return set_error(LQ_ERR_IO, "XML: unterminated comment");
            p = e + 3;
            continue;
        }
        if (s.compare(p, 13, "</parameters>") == 0 || s.compare(p, 12, "</parameters") == 0) break;
        if (s[p] != '<') return set_error(LQ_ERR_IO, "XML: unexpected text at offset %zu", p);
        size_t q = p + 1;
        while (q < s.size() && !is_space(s[q]) && s[q] != '>' && s[q] != '/') ++q;
        const std::string name = s.substr(p + 1, q - p - 1);
        size_t close = s.find('>', q);
        if (name.empty() || close == std::string::npos) return set_error(LQ_ERR_IO, "XML: malformed element");
        const std::string attrs = s.substr(q, close - q);
        if (!attrs.empty() && attrs.back() == '/')
            return set_error(LQ_ERR_IO, "XML: element %s has no value", name.c_str());
        std::string type;
        size_t t = attrs.find("type");
        if (t != std::string::npos) {
            size_t a = attrs.find_first_of("\"'", t);
            if (a != std::string::npos) {
                size_t b = attrs.find(attrs[a], a + 1);
                if (b != std::string::npos) type = attrs.substr(a + 1, b - a - 1);
            }
        }
        const std::string end_tag = "</" + name;
        size_t e = s.find(end_tag, close + 1);
        if (e == std::string::npos) return set_error(LQ_ERR_IO, "XML: element %s is not closed", name.c_str());
        std::string text = s.substr(close + 1, e - close - 1);
        size_t e2 = s.find('>', e);
        if (e2 == std::string::npos) return set_error(LQ_ERR_IO, "XML: malformed closing tag of %s", name.c_str());
        p = e2 + 1;
        XmlValue v{};
        if (type == "int") {
            v.is_int = true;
            v.i = atoi(text.c_str());
        } else if (type == "float") {
            v.is_int = false;
            v.f = (float)atof(text.c_str());
        } else {
            /* reference src/loquat_io.cu:111-114 */
            return set_error(LQ_ERR_IO, "XML: wrong data type for %s", name.c_str());
        }
        kv[name] = v;
    }
    return LQ_OK;
}

struct Reader {
    const std::map<std::string, XmlValue>& kv;
    int status = LQ_OK;
    int get_int(const char* key)
    {
        if (status != LQ_OK) return 0;
        auto it = kv.find(key);
        if (it == kv.end()) {
            status = set_error(LQ_ERR_NOTFOUND, "%s does not exist in the xml file", key);
            return 0;
        }
        if (!it->second.is_int) {
            status = set_error(LQ_ERR_IO, "%s must have type=\"int\"", key);
            return 0;
        }
        return it->second.i;
    }
    float get_float(const char* key)
    {
        if (status != LQ_OK) return 0.0f;
        auto it = kv.find(key);
        if (it == kv.end()) {
            status = set_error(LQ_ERR_NOTFOUND, "%s does not exist in the xml file", key);
            return 0.0f;
        }
        if (it->second.is_int) {
            status = set_error(LQ_ERR_IO, "%s must have type=\"float\"", key);
            return 0.0f;
        }
        return it->second.f;
    }
};

std::string fmt_float(float v)
{
    char buf[64];
    auto r = std::to_chars(buf, buf + sizeof(buf), v);
    return std::string(buf, r.ptr);
}

}  // namespace

extern "C" int lq_io_load_parameters(const char* xml_path, void* par_host)
{
    if (!xml_path || !par_host) return set_error(LQ_ERR_ARG, "lq_io_load_parameters: null argument");
    std::string text;
    if (!read_file(xml_path, text)) return set_error(LQ_ERR_IO, "cannot load the parameter file %s", xml_path);
    std::map<std::string, XmlValue> kv;
    LQ_TRY(parse_parameters_xml(text, kv));
    Reader r{kv};
    Parameters p;
    memset(&p, 0, sizeof(p));
    p.np = r.get_int("number-of-particles");
    p.npb = r.get_int("number-of-boundary-particles");
    p.npm = r.get_int("number-of-material-particles");
    if (r.status == LQ_OK && p.np != p.npb + p.npm)
        return set_error(LQ_ERR_IO, "wrong number of particles: %d != %d + %d", p.np, p.npb, p.npm);
    p.domain_size_x = r.get_float("domain-size-x");
    p.domain_size_y = r.get_float("domain-size-y");
    p.domain_size_z = r.get_float("domain-size-z");
    p.domain_min_x = r.get_float("domain-min-x");
    p.domain_min_y = r.get_float("domain-min-y");
    p.domain_min_z = r.get_float("domain-min-z");
    p.dr = r.get_float("particle-size");
    p.hdr = r.get_float("h-over-dr");
    p.rho0 = r.get_float("reference-density");
    p.cs = r.get_float("speed-of-sound");
    p.cfl = r.get_float("cfl-number");
    p.constitutive_model = r.get_int("constitutive-model");
    if (p.constitutive_model == 1) {
        p.model_par_1 = r.get_float("elastic-K");
        p.model_par_2 = r.get_float("elastic-G");
        p.model_par_3 = r.get_float("DP-kphi");
        p.model_par_4 = r.get_float("DP-kpsi");
        p.model_par_5 = r.get_float("DP-kcohesion");
    } else if (p.constitutive_model == 2) {
        p.model_par_1 = r.get_float("hypo-par-c1");
        p.model_par_2 = r.get_float("hypo-par-c2");
        p.model_par_3 = r.get_float("hypo-par-c3");
        p.model_par_4 = r.get_float("hypo-par-c4");
        p.model_par_5 = r.get_float("cohesion");
    }
    p.acc_x = r.get_float("acceleration-x");
    p.acc_y = r.get_float("acceleration-y");
    p.acc_z = r.get_float("acceleration-z");
    p.time_max = r.get_float("time-max");
    p.time = r.get_float("time");
    p.dt = r.get_float("time-step");
    p.output_frequency = r.get_float("output-frequency");
    p.output_number = r.get_int("output-number");
    p.density_shepard_filter = r.get_int("density-shepard-filter");
    p.stress_shepard_filter = r.get_int("stress-shepard-filter");
    p.dynamic_time_step = r.get_int("dynamic-time-step");
    p.integration_method = r.get_int("integration-method");
    p.viscosity_type = r.get_int("viscosity-type");
    if (p.viscosity_type == 1) p.artificial_viscosity_alpha = r.get_float("artificial-viscosity-alpha");
    p.artificial_pressure = r.get_int("artificial-pressure");
    if (p.artificial_pressure == 1) p.artificial_pressure_coefficient = r.get_float("artificial-pressure-coefficient");
    p.output_format = r.get_int("output-format");
    if (r.status != LQ_OK) return r.status;
    memcpy(par_host, &p, sizeof(p));
    return LQ_OK;
}

namespace {

/* Keys of constitutive model 3 (von Wolffersdorff), an extension with no
 * counterpart in the reference's parameter file: the 10-float material row
 * of lq_sim_set_hypoplastic and the initial void ratio. */
const char* const kVwKeys[9] = {"vw-phi-c", "vw-hs", "vw-n", "vw-ed0", "vw-ec0", "vw-ei0", "vw-alpha", "vw-beta",
                                "vw-tolerance"};
const char* const kVwMaxSub = "vw-max-substeps";
const char* const kVwE0 = "vw-initial-void-ratio";

/* Writes the parameter file; `vw` (10 floats) and e0 add the model-3 keys. */
int write_parameters(const char* xml_path, const Parameters& p, const float* vw, float e0)
{
    FILE* fp = fopen(xml_path, "w");
    if (!fp) return set_error(LQ_ERR_IO, "cannot write file %s", xml_path);
    auto I = [&](const char* k, int v) { fprintf(fp, "  <%s type=\"int\">%d</%s>\n", k, v, k); };
    auto F = [&](const char* k, float v) { fprintf(fp, "  <%s type=\"float\">%s</%s>\n", k, fmt_float(v).c_str(), k); };
    fprintf(fp, "<?xml version=\"1.0\" encoding=\"utf-8\" ?>\n<parameters>\n");
    I("number-of-particles", p.np);
    I("number-of-boundary-particles", p.npb);
    I("number-of-material-particles", p.npm);
    F("domain-size-x", p.domain_size_x);
    F("domain-size-y", p.domain_size_y);
    F("domain-size-z", p.domain_size_z);
    F("domain-min-x", p.domain_min_x);
    F("domain-min-y", p.domain_min_y);
    F("domain-min-z", p.domain_min_z);
    F("particle-size", p.dr);
    F("h-over-dr", p.hdr);
    F("reference-density", p.rho0);
    F("speed-of-sound", p.cs);
    F("cfl-number", p.cfl);
    I("constitutive-model", p.constitutive_model);
    if (p.constitutive_model == 1) {
        F("elastic-K", p.model_par_1);
        F("elastic-G", p.model_par_2);
        F("DP-kphi", p.model_par_3);
        F("DP-kpsi", p.model_par_4);
        F("DP-kcohesion", p.model_par_5);
    } else if (p.constitutive_model == 2) {
        F("hypo-par-c1", p.model_par_1);
        F("hypo-par-c2", p.model_par_2);
        F("hypo-par-c3", p.model_par_3);
        F("hypo-par-c4", p.model_par_4);
        F("cohesion", p.model_par_5);
    }
    F("acceleration-x", p.acc_x);
    F("acceleration-y", p.acc_y);
    F("acceleration-z", p.acc_z);
    F("time-max", p.time_max);
    F("time", p.time);
    F("time-step", p.dt);
    F("output-frequency", p.output_frequency);
    I("output-number", p.output_number);
    I("density-shepard-filter", p.density_shepard_filter);
    I("stress-shepard-filter", p.stress_shepard_filter);
    I("dynamic-time-step", p.dynamic_time_step);
    I("integration-method", p.integration_method);
    I("viscosity-type", p.viscosity_type);
    if (p.viscosity_type == 1) F("artificial-viscosity-alpha", p.artificial_viscosity_alpha);
    I("artificial-pressure", p.artificial_pressure);
    if (p.artificial_pressure == 1) F("artificial-pressure-coefficient", p.artificial_pressure_coefficient);
    I("output-format", p.output_format);
    if (vw) {
        for (int k = 0; k < 9; ++k) F(kVwKeys[k], vw[k]);
        I(kVwMaxSub, (int)vw[9]);
        F(kVwE0, e0);
    }
    fprintf(fp, "</parameters>\n");
    const bool ok = ferror(fp) == 0;
    fclose(fp);
    return ok ? LQ_OK : set_error(LQ_ERR_IO, "write error on %s", xml_path);
}

}  // namespace

extern "C" int lq_io_save_parameters(const char* xml_path, const void* par_host)
{
    if (!xml_path || !par_host) return set_error(LQ_ERR_ARG, "lq_io_save_parameters: null argument");
    return write_parameters(xml_path, *static_cast<const Parameters*>(par_host), nullptr, 0.0f);
}

extern "C" int lq_io_save_parameters_vw(const char* xml_path, const void* par_host, const float* vw_row, float e0)
{
    if (!xml_path || !par_host || !vw_row) return set_error(LQ_ERR_ARG, "lq_io_save_parameters_vw: null argument");
    return write_parameters(xml_path, *static_cast<const Parameters*>(par_host), vw_row, e0);
}

extern "C" int lq_io_load_hypoplastic(const char* xml_path, float* vw_row, float* e0)
{
    if (!xml_path || !vw_row || !e0) return set_error(LQ_ERR_ARG, "lq_io_load_hypoplastic: null argument");
    std::string text;
    if (!read_file(xml_path, text)) return set_error(LQ_ERR_IO, "cannot load the parameter file %s", xml_path);
    std::map<std::string, XmlValue> kv;
    LQ_TRY(parse_parameters_xml(text, kv));
    Reader r{kv};
    float row[10];
    for (int k = 0; k < 9; ++k) row[k] = r.get_float(kVwKeys[k]);
    row[9] = (float)r.get_int(kVwMaxSub);
    const float v = r.get_float(kVwE0);
    if (r.status != LQ_OK) return r.status;
    memcpy(vw_row, row, sizeof(row));
    *e0 = v;
    return LQ_OK;
}

extern "C" int lq_io_load_particles(const char* dat_path, int np, float* pos, float* vel, float* idep, float* str,
                                    float* stn)
{
    if (!dat_path || np < 0 || (np > 0 && (!pos || !vel || !idep || !str || !stn)))
        return set_error(LQ_ERR_ARG, "lq_io_load_particles: bad argument");
    std::string text;
    if (!read_file(dat_path, text)) return set_error(LQ_ERR_IO, "cannot open %s", dat_path);
    const char* c = text.c_str();
    const char* end = c + text.size();
    float row[22];
    for (int i = 0; i < np; ++i) {
        for (int k = 0; k < 22; ++k) {
            while (c < end && is_space(*c)) ++c;
            if (c >= end)
                return set_error(LQ_ERR_IO, "%s: truncated at particle %d column %d (expected %d particles)", dat_path,
                                 i, k, np);
            char* next = nullptr;
            errno = 0;
            row[k] = strtof(c, &next);
            if (next == c) return set_error(LQ_ERR_IO, "%s: not a number at particle %d column %d", dat_path, i, k);
            c = next;
        }
        float* P = pos + 4 * (size_t)i;
        float* V = vel + 4 * (size_t)i;
        float* D = idep + 4 * (size_t)i;
        float* S = str + 6 * (size_t)i;
        float* E = stn + 6 * (size_t)i;
        for (int k = 0; k < 4; ++k) P[k] = row[k];
        for (int k = 0; k < 4; ++k) V[k] = row[4 + k];
        D[0] = row[8];
        D[1] = row[9];
        D[2] = 0.0f;
        D[3] = 0.0f;
        for (int k = 0; k < 6; ++k) S[k] = row[10 + k];
        for (int k = 0; k < 6; ++k) E[k] = row[16 + k];
    }
    return LQ_OK;
}

extern "C" int lq_io_save_particles(const char* dat_path, int np, const float* pos, const float* vel,
                                    const float* idep, const float* str, const float* stn)
{
    if (!dat_path || np < 0 || (np > 0 && (!pos || !vel || !idep || !str || !stn)))
        return set_error(LQ_ERR_ARG, "lq_io_save_particles: bad argument");
    FILE* fp = fopen(dat_path, "w");
    if (!fp) return set_error(LQ_ERR_IO, "cannot write in %s", dat_path);
    std::vector<char> line(22 * 20 + 8);
    for (int i = 0; i < np; ++i) {
        float row[22];
        const float* P = pos + 4 * (size_t)i;
        const float* V = vel + 4 * (size_t)i;
        const float* D = idep + 4 * (size_t)i;
        const float* S = str + 6 * (size_t)i;
        const float* E = stn + 6 * (size_t)i;
        for (int k = 0; k < 4; ++k) row[k] = P[k];
        for (int k = 0; k < 4; ++k) row[4 + k] = V[k];
        row[8] = D[0];
        row[9] = D[1];
        for (int k = 0; k < 6; ++k) row[10 + k] = S[k];
        for (int k = 0; k < 6; ++k) row[16 + k] = E[k];
        char* w = line.data();
        char* lim = w + line.size();
        for (int k = 0; k < 22; ++k) {
            auto r = std::to_chars(w, lim, row[k]);
            w = r.ptr;
            *w++ = (k == 21) ? '\n' : ' ';
        }
        fwrite(line.data(), 1, (size_t)(w - line.data()), fp);
    }
    const bool ok = ferror(fp) == 0;
    fclose(fp);
    return ok ? LQ_OK : set_error(LQ_ERR_IO, "write error on %s", dat_path);
}

/* ParaView output (reference src/loquat_io.cu:372-548): one ASCII .vtu file
 * per object id, "<dir>/<id>_<n>.vtu", objects in descending id order, each
 * a piece of vertex cells with Pressure, Velocity, Density, PlasticStrain,
 * Stress, Strain point data. */
extern "C" int lq_io_save_vtu(const char* dir, int output_number, int np, const float* pos, const float* vel,
                              const float* idep, const float* str, const float* stn)
{
    if (!dir || np < 0 || (np > 0 && (!pos || !vel || !idep || !str || !stn)))
        return set_error(LQ_ERR_ARG, "lq_io_save_vtu: bad argument");
    std::vector<int> order(np);
    for (int i = 0; i < np; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        return (int)idep[4 * (size_t)a] > (int)idep[4 * (size_t)b];
    });
    size_t k = 0;
    char buf[64];
    auto put = [&](FILE* fp, float v) {
        auto r = std::to_chars(buf, buf + sizeof(buf), v);
        *r.ptr++ = ' ';
        fwrite(buf, 1, (size_t)(r.ptr - buf), fp);
    };
    while (k < order.size()) {
        const int id = (int)idep[4 * (size_t)order[k]];
        size_t e = k;
        while (e < order.size() && (int)idep[4 * (size_t)order[e]] == id) ++e;
        const size_t n = e - k;
        std::string name = std::string(dir) + "/" + std::to_string(id) + "_" + std::to_string(output_number) + ".vtu";
        FILE* fp = fopen(name.c_str(), "w");
        if (!fp) return set_error(LQ_ERR_IO, "cannot write file %s", name.c_str());
        fprintf(fp, "<?xml version=\"1.0\"?>\n<VTKFile type=\"UnstructuredGrid\" version=\"0.1\" "
                    "byte_order=\"LittleEndian\">\n  <UnstructuredGrid GhostLevel=\"0\">\n"
                    "    <Piece NumberOfPoints=\"%zu\" NumberOfCells=\"%zu\" Name=\"%d\">\n      <PointData>\n",
                n, n, id);
        auto arr = [&](const char* label, int comps, auto getter) {
            if (comps > 1)
                fprintf(fp, "        <DataArray type=\"Float32\" Name=\"%s\" NumberOfComponents=\"%d\">\n", label,
                        comps);
            else
                fprintf(fp, "        <DataArray type=\"Float32\" Name=\"%s\">\n", label);
            for (size_t q = k; q < e; ++q) getter((size_t)order[q], fp);
            fprintf(fp, "</DataArray>\n");
        };
        arr("Pressure", 1, [&](size_t i, FILE* f) { put(f, pos[4 * i + 3]); });
        arr("Velocity", 3, [&](size_t i, FILE* f) { for (int c = 0; c < 3; ++c) put(f, vel[4 * i + c]); });
        arr("Density", 1, [&](size_t i, FILE* f) { put(f, vel[4 * i + 3]); });
        arr("PlasticStrain", 1, [&](size_t i, FILE* f) { put(f, idep[4 * i + 1]); });
        arr("Stress", 6, [&](size_t i, FILE* f) { for (int c = 0; c < 6; ++c) put(f, str[6 * i + c]); });
        arr("Strain", 6, [&](size_t i, FILE* f) { for (int c = 0; c < 6; ++c) put(f, stn[6 * i + c]); });
        fprintf(fp, "      </PointData>\n      <CellData>\n      </CellData>\n      <Points>\n");
        arr("Points", 3, [&](size_t i, FILE* f) { for (int c = 0; c < 3; ++c) put(f, pos[4 * i + c]); });
        fprintf(fp, "      </Points>\n      <Cells>\n");
        fprintf(fp, "        <DataArray type=\"Int64\" Name=\"connectivity\" format=\"ascii\">\n");
        for (size_t q = 0; q < n; ++q) fprintf(fp, "%zu ", q);
        fprintf(fp, "</DataArray>\n        <DataArray type=\"Int64\" Name=\"offsets\" format=\"ascii\">\n");
        for (size_t q = 0; q < n; ++q) fprintf(fp, "%zu ", q + 1);
        fprintf(fp, "</DataArray>\n        <DataArray type=\"Int64\" Name=\"types\" format=\"ascii\">\n");
        for (size_t q = 0; q < n; ++q) fputs("1 ", fp);
        fprintf(fp, "</DataArray>\n      </Cells>\n    </Piece>\n  </UnstructuredGrid>\n</VTKFile>\n");
        const bool ok = ferror(fp) == 0;
        fclose(fp);
        if (!ok) return set_error(LQ_ERR_IO, "write error on %s", name.c_str());
        k = e;
    }
    return LQ_OK;
}
