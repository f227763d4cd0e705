// Host-side geometry: a small XML reader for the Kerkythea scene format,
// the box voxeliser, material coefficient files and the LRS classification.
#include "model.hpp"

#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <set>
#include <sstream>

#include "../../include/afd.h"

namespace afd {

// ---------------------------------------------------------------------------
// Minimal XML reader: elements, attributes, comments, processing
// instructions, DOCTYPE and CDATA (skipped). Text content is ignored; the
// scene format keeps all data in attributes.
// ---------------------------------------------------------------------------
namespace {

struct XNode {
    std::string name;
    std::vector<std::pair<std::string, std::string>> attrs;
    std::vector<XNode> kids;

    const std::string* attr(const char* key) const {
        for (auto& kv : attrs)
            if (kv.first == key) return &kv.second;
        return nullptr;
    }
    std::string attr_or_empty(const char* key) const {
        const std::string* v = attr(key);
        return v ? *v : std::string();
    }
    const XNode* first_child(const char* nm) const {
        for (auto& k : kids)
            if (k.name == nm) return &k;
        return nullptr;
    }
};

class XmlReader {
public:
    explicit XmlReader(const std::string& text) : s_(text), i_(0) {}

    XNode parse_document() {
        XNode doc;
        doc.name = "#document";
        parse_content(doc, /*top=*/true);
        return doc;
    }

private:
    const std::string& s_;
    size_t i_;

    [[noreturn]] void fail(const char* what) {
        throw Error(AFD_ERR_IO, std::string("XML parse error: ") + what + " at byte " +
                                    std::to_string(i_));
    }
    bool starts(const char* lit) const { return s_.compare(i_, std::strlen(lit), lit) == 0; }
    void skip_until(const char* lit) {
        size_t p = s_.find(lit, i_);
        if (p == std::string::npos) fail("unterminated construct");
        i_ = p + std::strlen(lit);
    }
    static bool is_space(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r'; }
    static bool is_name_char(char c) {
        return !(is_space(c) || c == '=' || c == '>' || c == '/' || c == '<' || c == '"' ||
                 c == '\'' || c == '\0');
    }
    void skip_ws() {
        while (i_ < s_.size() && is_space(s_[i_])) ++i_;
    }
    std::string read_name() {
        size_t b = i_;
        while (i_ < s_.size() && is_name_char(s_[i_])) ++i_;
        if (b == i_) fail("expected a name");
        return s_.substr(b, i_ - b);
    }
    static void put_utf8(std::string& out, unsigned long cp) {
        if (cp < 0x80) {
            out += (char)cp;
        } else if (cp < 0x800) {
            out += (char)(0xC0 | (cp >> 6));
            out += (char)(0x80 | (cp & 0x3F));
        } else if (cp < 0x10000) {
            out += (char)(0xE0 | (cp >> 12));
            out += (char)(0x80 | ((cp >> 6) & 0x3F));
            out += (char)(0x80 | (cp & 0x3F));
        } else {
            out += (char)(0xF0 | (cp >> 18));
            out += (char)(0x80 | ((cp >> 12) & 0x3F));
            out += (char)(0x80 | ((cp >> 6) & 0x3F));
            out += (char)(0x80 | (cp & 0x3F));
        }
    }
    // Attribute values: entity references decoded, tab/CR/LF read as spaces.
    static std::string decode(const std::string& raw) {
        std::string out;
        out.reserve(raw.size());
        for (size_t k = 0; k < raw.size(); ++k) {
            char c = raw[k];
            if (c == '&') {
                size_t semi = raw.find(';', k);
                if (semi != std::string::npos) {
                    std::string ent = raw.substr(k + 1, semi - k - 1);
                    bool ok = true;
                    if (ent == "lt") out += '<';
                    else if (ent == "gt") out += '>';
                    else if (ent == "amp") out += '&';
                    else if (ent == "apos") out += '\'';
                    else if (ent == "quot") out += '"';
                    else if (ent.size() > 1 && ent[0] == '#') {
                        unsigned long cp = (ent[1] == 'x' || ent[1] == 'X')
                                               ? std::strtoul(ent.c_str() + 2, nullptr, 16)
                                               : std::strtoul(ent.c_str() + 1, nullptr, 10);
                        put_utf8(out, cp);
                    } else {
                        ok = false;
                    }
                    if (ok) {
                        k = semi;
                        continue;
                    }
                }
                out += c;
            } else if (c == '\t' || c == '\n' || c == '\r') {
                out += ' ';
            } else {
                out += c;
            }
        }
        return out;
    }

    // Parses children until the parent's end tag (or end of input at top level).
    void parse_content(XNode& parent, bool top) {
        while (true) {
            size_t lt = s_.find('<', i_);
            if (lt == std::string::npos) {
                if (!top) fail("missing end tag");
                i_ = s_.size();
                return;
            }
            i_ = lt;
            if (starts("<!--")) {
                skip_until("-->");
            } else if (starts("<![CDATA[")) {
                skip_until("]]>");
            } else if (starts("<?")) {
                skip_until("?>");
            } else if (starts("<!")) {
                skip_until(">");
            } else if (starts("</")) {
                if (top) fail("unexpected end tag");
                i_ += 2;
                std::string nm = read_name();
                if (nm != parent.name) fail("mismatched end tag");
                skip_ws();
                if (i_ >= s_.size() || s_[i_] != '>') fail("bad end tag");
                ++i_;
                return;
            } else {
                ++i_;
                XNode node;
                node.name = read_name();
                bool closed = false;
                while (true) {
                    skip_ws();
                    if (i_ >= s_.size()) fail("unterminated tag");
                    if (s_[i_] == '/') {
                        if (i_ + 1 >= s_.size() || s_[i_ + 1] != '>') fail("bad empty tag");
                        i_ += 2;
                        closed = true;
                        break;
                    }
                    if (s_[i_] == '>') {
                        ++i_;
                        break;
                    }
                    std::string key = read_name();
                    skip_ws();
                    if (i_ >= s_.size() || s_[i_] != '=') fail("expected '='");
                    ++i_;
                    skip_ws();
                    if (i_ >= s_.size() || (s_[i_] != '"' && s_[i_] != '\'')) fail("expected quote");
                    char q = s_[i_++];
                    size_t end = s_.find(q, i_);
                    if (end == std::string::npos) fail("unterminated attribute");
                    node.attrs.emplace_back(key, decode(s_.substr(i_, end - i_)));
                    i_ = end + 1;
                }
                if (!closed) parse_content(node, false);
                parent.kids.push_back(std::move(node));
            }
        }
    }
};

std::string read_file(const std::string& path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw Error(AFD_ERR_IO, "cannot open " + path);
    std::ostringstream ss;
    ss << f.rdbuf();
    return ss.str();
}

// Parses "%f %f %f" as sscanf does (strtof per field).
bool parse_three_floats(const std::string& s, float v[3]) {
    const char* p = s.c_str();
    for (int k = 0; k < 3; ++k) {
        char* end = nullptr;
        errno = 0;
        float f = std::strtof(p, &end);
        if (end == p) return false;
        v[k] = f;
        p = end;
    }
    return true;
}

// Util::GetDirectory (util.hpp:117-122), except that a bare file name maps to
// the current directory instead of to itself.
std::string directory_of(const std::string& path) {
    size_t found = path.find_last_of("/\\");
    if (found == std::string::npos) return ".";
    return path.substr(0, found);
}

}  // namespace

std::vector<Box> load_boxes(const std::string& xml_path) {
    std::string text = read_file(xml_path);
    XNode doc = XmlReader(text).parse_document();
    std::vector<Box> boxes;
    const XNode* root = doc.first_child("Root");
    if (!root) return boxes;
    for (const XNode& scene : root->kids) {
        if (scene.name != "Object" || scene.attr_or_empty("Type") != "Scene") continue;
        for (const XNode& model : scene.kids) {
            if (model.name != "Object" || model.attr_or_empty("Type") != "Model") continue;
            std::string name = model.attr_or_empty("Name");
            const XNode* surf = model.first_child("Object");
            if (!surf) continue;
            for (const XNode& prm : surf->kids) {
                if (prm.name != "Parameter" || prm.attr_or_empty("Name") != "Vertex List") continue;
                float min_x = 10000.0f, min_y = 10000.0f, min_z = 10000.0f;
                float max_x = -10000.0f, max_y = -10000.0f, max_z = -10000.0f;
                int npts = 0;
                for (const XNode& pt : prm.kids) {
                    if (pt.name != "P") continue;
                    float abc[3];
                    if (!parse_three_floats(pt.attr_or_empty("xyz"), abc))
                        throw Error(AFD_ERR_IO, "bad vertex in model " + name);
                    // Axis remap (x, y, z) <- (a, c, -b), kerkythea.hpp:97-99.
                    float x = abc[0], y = abc[2], z = -abc[1];
                    if (x < min_x) min_x = x;
                    if (x > max_x) max_x = x;
                    if (y < min_y) min_y = y;
                    if (y > max_y) max_y = y;
                    if (z < min_z) min_z = z;
                    if (z > max_z) max_z = z;
                    ++npts;
                }
                if (npts == 0) continue;  // an empty vertex list describes no box
                std::string mat = name.substr(name.find_last_of('_') + 1);
                if (min_x < 0.0f) min_x = 0.0f;
                if (min_y < 0.0f) min_y = 0.0f;
                if (min_z < 0.0f) min_z = 0.0f;
                boxes.push_back(Box{{min_x, max_x, min_y, max_y, min_z, max_z}, mat});
            }
        }
    }
    return boxes;
}

std::vector<float> read_coefficients(const std::string& path) {
    std::ifstream f(path);
    if (!f) throw Error(AFD_ERR_IO, "cannot open coefficient file " + path);
    std::vector<float> out;
    std::string line;
    while (std::getline(f, line)) {
        const char* p = line.c_str();
        char* end = nullptr;
        double v = std::strtod(p, &end);
        if (end == p) throw Error(AFD_ERR_IO, "bad coefficient line in " + path + ": '" + line + "'");
        out.push_back((float)v);
    }
    if (out.empty()) throw Error(AFD_ERR_IO, "empty coefficient file " + path);
    return out;
}

Scene parse_kerkythea(const std::string& xml_path, float res) {
    if (!(res > 0.0f)) throw Error(AFD_ERR_ARG, "cell size must be positive");
    std::vector<Box> boxes = load_boxes(xml_path);
    if (boxes.empty()) throw Error(AFD_ERR_IO, "no boxes found in " + xml_path);

    float max_x = 0.0f, max_y = 0.0f, max_z = 0.0f;
    for (auto& b : boxes) {
        if (b.ext[1] > max_x) max_x = b.ext[1];
        if (b.ext[3] > max_y) max_y = b.ext[3];
        if (b.ext[5] > max_z) max_z = b.ext[5];
    }
    Scene sc;
    Model& m = sc.model;
    m.nx = (int32_t)round_to((uint32_t)(cell_of(max_x, res) + 1), 32);
    m.ny = (int32_t)round_to((uint32_t)(cell_of(max_y, res) + 1), 32);
    m.nz = (int32_t)round_to((uint32_t)(cell_of(max_z, res) + 1), 32);

    std::set<std::string> names;
    for (auto& b : boxes) names.insert(b.material);
    std::string dir = directory_of(xml_path);
    std::map<std::string, int32_t> index;
    for (const std::string& nm : names) {
        std::vector<float> ca = read_coefficients(dir + "/" + nm + "_a.dat");
        std::vector<float> cb = read_coefficients(dir + "/" + nm + "_b.dat");
        if (m.material_names.empty()) m.ncoef = (int32_t)ca.size();
        if ((int32_t)ca.size() != m.ncoef || (int32_t)cb.size() != m.ncoef)
            throw Error(AFD_ERR_IO, "material " + nm + " has a filter order different from " +
                                        *names.begin());
        m.a.insert(m.a.end(), ca.begin(), ca.end());
        m.b.insert(m.b.end(), cb.begin(), cb.end());
        index[nm] = (int32_t)m.material_names.size();
        m.material_names.push_back(nm);
    }
    m.nmat = (int32_t)m.material_names.size();

    // Cell ranges of the boxes in file order (kerkythea.hpp:180-195). A box
    // whose maximum lies below zero on some axis covers no cell; the minimum
    // was clamped at zero, and the grid ends past every maximum's cell, so
    // every range lies inside the grid.
    for (auto& b : boxes) {
        if (b.ext[1] < 0.0f || b.ext[3] < 0.0f || b.ext[5] < 0.0f) continue;
        BoxCells c;
        const int32_t n[3] = {m.nx, m.ny, m.nz};
        for (int k = 0; k < 3; ++k) {
            c.lo[k] = (int32_t)cell_of(b.ext[2 * k], res);
            c.hi[k] = (int32_t)cell_of(b.ext[2 * k + 1], res);
            if (c.lo[k] < 0 || c.hi[k] >= n[k]) throw Error(AFD_ERR_IO, "box outside the grid in " + xml_path);
        }
        c.mat = index.at(b.material);
        sc.boxes.push_back(c);
    }
    return sc;
}

void rasterize_host(const Scene& sc, Model& m) {
    m.vox.assign((size_t)m.cells(), -1);
    // inclusive ranges, later boxes overwrite earlier ones
    for (const BoxCells& c : sc.boxes)
        for (int64_t z = c.lo[2]; z <= c.hi[2]; ++z)
            for (int64_t y = c.lo[1]; y <= c.hi[1]; ++y)
                for (int64_t x = c.lo[0]; x <= c.hi[0]; ++x) m.vox[(size_t)((z * m.ny + y) * m.nx + x)] = c.mat;
}

Model load_kerkythea(const std::string& xml_path, float res) {
    Scene sc = parse_kerkythea(xml_path, res);
    Model m = std::move(sc.model);
    rasterize_host(sc, m);
    return m;
}

const uint8_t kGroupMask[kNumGroups] = {
    1u << DXP, 1u << DXM, 1u << DYP, 1u << DYM, 1u << DZP, 1u << DZM,
    (1u << DXP) | (1u << DYP), (1u << DXP) | (1u << DYM),
    (1u << DXP) | (1u << DZP), (1u << DXP) | (1u << DZM),
    (1u << DXM) | (1u << DYP), (1u << DXM) | (1u << DYM),
    (1u << DXM) | (1u << DZP), (1u << DXM) | (1u << DZM),
    (1u << DYP) | (1u << DZP), (1u << DYP) | (1u << DZM),
    (1u << DYM) | (1u << DZP), (1u << DYM) | (1u << DZM),
    (1u << DXP) | (1u << DYP) | (1u << DZP), (1u << DXP) | (1u << DYP) | (1u << DZM),
    (1u << DXP) | (1u << DYM) | (1u << DZP), (1u << DXP) | (1u << DYM) | (1u << DZM),
    (1u << DXM) | (1u << DYP) | (1u << DZP), (1u << DXM) | (1u << DYP) | (1u << DZM),
    (1u << DXM) | (1u << DYM) | (1u << DZP), (1u << DXM) | (1u << DYM) | (1u << DZM),
};

int group_faces(int g) { return g < 6 ? 1 : (g < 18 ? 2 : 3); }

int group_of_mask(unsigned mask) {
    for (int g = 0; g < kNumGroups; ++g)
        if (kGroupMask[g] == mask) return g;
    return -1;
}

std::vector<BoundaryPoint> classify(const Model& m) {
    std::vector<BoundaryPoint> pts;
    const int64_t nx = m.nx, ny = m.ny, nz = m.nz;
    const int32_t* v = m.vox.data();
    auto V = [&](int64_t x, int64_t y, int64_t z) { return v[(z * ny + y) * nx + x]; };
    for (int64_t z = 1; z < nz - 1; ++z)
        for (int64_t y = 1; y < ny - 1; ++y)
            for (int64_t x = 1; x < nx - 1; ++x) {
                if (V(x, y, z) != -1) continue;
                int32_t nb[6] = {V(x + 1, y, z), V(x - 1, y, z), V(x, y + 1, z),
                                 V(x, y - 1, z), V(x, y, z + 1), V(x, y, z - 1)};
                unsigned mask = 0;
                for (int d = 0; d < 6; ++d)
                    if (nb[d] != -1) mask |= 1u << d;
                if (!mask) continue;
                int g = group_of_mask(mask);
                if (g < 0) {
                    char buf[160];
                    std::snprintf(buf, sizeof buf,
                                  "Unphysical surfaces encountered at cell (%lld,%lld,%lld)",
                                  (long long)x, (long long)y, (long long)z);
                    throw Error(AFD_ERR_GEOMETRY, buf);
                }
                BoundaryPoint p{(int32_t)x, (int32_t)y, (int32_t)z, g, {-1, -1, -1}};
                int k = 0;
                for (int d = 0; d < 6; ++d)
                    if (mask & (1u << d)) p.mat[k++] = nb[d];
                pts.push_back(p);
            }
    return pts;
}

std::vector<float> load_text_matrix(const std::string& path, int64_t* rows, int64_t* cols) {
    std::ifstream f(path);
    if (!f) throw Error(AFD_ERR_IO, "cannot open " + path);
    std::vector<float> out;
    std::string line, tok;
    int64_t r = 0, c0 = -1;
    while (std::getline(f, line)) {
        std::istringstream ss(line);
        int64_t c = 0;
        while (ss >> tok) {
            out.push_back((float)std::atof(tok.c_str()));
            ++c;
        }
        if (c0 < 0) c0 = c;
        else if (c != c0)
            throw Error(AFD_ERR_IO, "row " + std::to_string(r) + " of " + path +
                                        " has a different length than the first row");
        ++r;
    }
    if (rows) *rows = r;
    if (cols) *cols = c0 < 0 ? 0 : c0;
    return out;
}

void save_rows(const std::string& path, const float* data, int64_t rows, int64_t cols) {
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) throw Error(AFD_ERR_IO, "cannot write " + path);
    std::vector<char> buf(1 << 20);
    std::setvbuf(f, buf.data(), _IOFBF, buf.size());
    for (int64_t j = 0; j < rows; ++j) {
        for (int64_t i = 0; i < cols; ++i) std::fprintf(f, "%.6g ", (double)data[j * cols + i]);
        std::fputc('\n', f);
    }
    std::fputc('\n', f);
    if (std::fclose(f) != 0) throw Error(AFD_ERR_IO, "write failed: " + path);
}

}  // namespace afd
