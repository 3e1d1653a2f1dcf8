// calib_xml.cpp -- intrinsics.xml and CalibInfo.xml (include/pfd_calib.h).
//
// A small XML reader (elements, attributes, text, comments, declarations, the
// five predefined entities) with tinyxml2's notion of an element's text: the
// first child when that child is a non-blank text node.  The field parses
// restate DepthSolver::ReadIntrinsicsFromXML (DepthSolver.cpp:872-1110) and
// ReadCalibrationParamsFromXML (:1112-1250); the writer restates
// WriteCalibrationParamsXML (:1252-1340).
#include <cctype>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <sstream>
#include <string>
#include <utility>
#include <vector>

#include "../../include/pfd_calib.h"

namespace {

struct Node {
    std::string name;
    std::vector<std::pair<std::string, std::string>> attrs;
    bool has_text = false;      // first child is a non-blank text node
    std::string text;
    std::vector<Node> kids;

    const Node* first(const char* n) const
    {
        for (const Node& k : kids)
            if (k.name == n) return &k;
        return nullptr;
    }
    const char* attr(const char* n) const
    {
        for (const auto& a : attrs)
            if (a.first == n) return a.second.c_str();
        return nullptr;
    }
};

class Parser {
public:
    explicit Parser(const char* s) : p_(s) {}

    bool document(Node& root)
    {
        skip_misc();
        if (*p_ != '<') return false;
        if (!element(root, 0)) return false;
        skip_misc();
        return *p_ == '\0';
    }

private:
    const char* p_;

    void skip_ws()
    {
        while (*p_ && std::isspace((unsigned char)*p_)) ++p_;
    }
    bool skip_special()                      // comment, declaration, doctype, processing instruction
    {
        if (std::strncmp(p_, "<!--", 4) == 0) {
            const char* e = std::strstr(p_ + 4, "-->");
            if (!e) return false;
            p_ = e + 3;
            return true;
        }
        if (std::strncmp(p_, "<?", 2) == 0) {
            const char* e = std::strstr(p_ + 2, "?>");
            if (!e) return false;
            p_ = e + 2;
            return true;
        }
        if (std::strncmp(p_, "<!", 2) == 0 && std::strncmp(p_, "<![CDATA[", 9) != 0) {
            const char* e = std::strchr(p_ + 2, '>');
            if (!e) return false;
            p_ = e + 1;
            return true;
        }
        return false;
    }
    void skip_misc()
    {
        for (;;) {
            skip_ws();
            if (!skip_special()) return;
        }
    }
    static bool name_char(char c) { return std::isalnum((unsigned char)c) || c == '_' || c == '-' || c == '.' || c == ':'; }
    bool name(std::string& out)
    {
        const char* s = p_;
        while (name_char(*p_)) ++p_;
        out.assign(s, p_);
        return !out.empty();
    }
    static void decode(const char* s, const char* e, std::string& out)
    {
        out.clear();
        while (s < e) {
            if (*s == '&') {
                static const struct { const char* ent; char c; } k[] = {
                    { "&lt;", '<' }, { "&gt;", '>' }, { "&amp;", '&' }, { "&quot;", '"' }, { "&apos;", '\'' } };
                bool hit = false;
                for (const auto& x : k) {
                    const size_t l = std::strlen(x.ent);
                    if ((size_t)(e - s) >= l && std::strncmp(s, x.ent, l) == 0) {
                        out.push_back(x.c);
                        s += l;
                        hit = true;
                        break;
                    }
                }
                if (hit) continue;
            }
            out.push_back(*s++);
        }
    }
    bool element(Node& n, int depth)
    {
        if (depth > 64 || *p_ != '<') return false;
        ++p_;
        if (!name(n.name)) return false;
        for (;;) {
            skip_ws();
            if (*p_ == '/') {
                if (p_[1] != '>') return false;
                p_ += 2;
                return true;
            }
            if (*p_ == '>') {
                ++p_;
                break;
            }
            std::string an, av;
            if (!name(an)) return false;
            skip_ws();
            if (*p_ != '=') return false;
            ++p_;
            skip_ws();
            const char q = *p_;
            if (q != '"' && q != '\'') return false;
            const char* s = ++p_;
            while (*p_ && *p_ != q) ++p_;
            if (!*p_) return false;
            decode(s, p_, av);
            ++p_;
            n.attrs.emplace_back(an, av);
        }
        bool any_child = false;
        for (;;) {
            if (*p_ == '\0') return false;
            if (*p_ == '<') {
                if (p_[1] == '/') {
                    p_ += 2;
                    std::string close;
                    if (!name(close) || close != n.name) return false;
                    skip_ws();
                    if (*p_ != '>') return false;
                    ++p_;
                    return true;
                }
                if (std::strncmp(p_, "<![CDATA[", 9) == 0) {
                    const char* s = p_ + 9;
                    const char* e = std::strstr(s, "]]>");
                    if (!e) return false;
                    if (!any_child) { n.has_text = true; n.text.assign(s, e); }
                    any_child = true;
                    p_ = e + 3;
                    continue;
                }
                if (skip_special()) continue;
                n.kids.emplace_back();
                if (!element(n.kids.back(), depth + 1)) return false;
                any_child = true;
                continue;
            }
            const char* s = p_;
            while (*p_ && *p_ != '<') ++p_;
            bool blank = true;
            for (const char* c = s; c < p_; ++c)
                if (!std::isspace((unsigned char)*c)) { blank = false; break; }
            if (!blank) {
                if (!any_child) { n.has_text = true; decode(s, p_, n.text); }
                any_child = true;
            }
        }
    }
};

// sscanf-like conversions: a failed conversion leaves the target unchanged.
const char* ws(const char* s)
{
    while (*s && std::isspace((unsigned char)*s)) ++s;
    return s;
}
const char* scan_f(const char* s, float* v)
{
    if (!s) return nullptr;
    char* e = nullptr;
    const float x = std::strtof(ws(s), &e);
    if (e == ws(s)) return nullptr;
    *v = x;
    return e;
}
const char* scan_lf(const char* s, double* v)
{
    if (!s) return nullptr;
    char* e = nullptr;
    const double x = std::strtod(ws(s), &e);
    if (e == ws(s)) return nullptr;
    *v = x;
    return e;
}
const char* scan_int(const char* s, int* v, int base)
{
    if (!s) return nullptr;
    char* e = nullptr;
    const long x = std::strtol(ws(s), &e, base);
    if (e == ws(s)) return nullptr;
    *v = (int)x;
    return e;
}
// "%f,%f" / "%i,%i": the second conversion runs only when a comma follows the first
void scan_pair_f(const char* s, float* a, float* b)
{
    const char* e = scan_f(s, a);
    if (e && *e == ',') scan_f(e + 1, b);
}
void scan_pair_i(const char* s, int* a, int* b)
{
    const char* e = scan_int(s, a, 0);
    if (e && *e == ',') scan_int(e + 1, b, 0);
}

const char* text_of(const Node* n) { return (n && n->has_text) ? n->text.c_str() : nullptr; }

// the i-th child element (0-based), or null
const Node* child(const Node* n, size_t i) { return (n && i < n->kids.size()) ? &n->kids[i] : nullptr; }

}  // namespace

extern "C" pfd_status pfd_read_intrinsics_xml(const char* text, pfd_intrinsics* out)
{
    if (!text || !out) return PFD_EINVAL;
    std::memset(out, 0, sizeof(*out));
    Node root;
    if (!Parser(text).document(root) || root.name != "_") return PFD_EINVAL;
    for (const Node& g : root.kids) {
        if (g.name == "D") {
            if (!g.has_text) return PFD_EINVAL;
            scan_f(g.text.c_str(), &out->D);
        } else if (g.name == "d") {
            if (!g.has_text) return PFD_EINVAL;
            scan_f(g.text.c_str(), &out->d);
        } else if (g.name == "sensor") {
            for (const Node& e : g.kids) {
                if (e.name == "pose") {
                    for (const Node& c : e.kids) {
                        if (c.name == "rotation") {
                            // up to three "_" children, one column each (DepthSolver.cpp:913-975)
                            for (int col = 0; col < 3; ++col) {
                                const Node* cn = child(&c, (size_t)col);
                                if (!cn) break;
                                if (cn->name != "_") continue;
                                for (int row = 0; row < 3; ++row) {
                                    const char* t = text_of(child(cn, (size_t)row));
                                    if (!t) return PFD_EINVAL;
                                    scan_lf(t, &out->sensor_rotation[row * 3 + col]);
                                }
                            }
                        } else if (c.name == "translation") {
                            const Node* u = child(&c, 0);
                            if (u && u->name == "_")
                                for (int i = 0; i < 3; ++i) {
                                    const char* t = text_of(child(u, (size_t)i));
                                    if (!t) return PFD_EINVAL;
                                    scan_lf(t, &out->sensor_translate[i]);
                                }
                        }
                    }
                } else if (e.name == "scale") {
                    if (!e.has_text) return PFD_EINVAL;
                    scan_f(e.text.c_str(), &out->sensor_pixel_size);
                }
            }
        } else if (g.name == "main_lens") {
            for (const Node& e : g.kids)
                if (e.name == "f") {
                    if (!e.has_text) return PFD_EINVAL;
                    scan_f(e.text.c_str(), &out->mainlen_focal_length);
                }
        } else if (g.name == "mia") {
            for (const Node& e : g.kids) {
                if (e.name != "mesh") continue;
                for (const Node& c : e.kids) {
                    if (c.name == "height") {
                        if (!c.has_text) return PFD_EINVAL;
                        scan_int(c.text.c_str(), &out->mla_v_size, 10);
                    } else if (c.name == "width") {
                        if (!c.has_text) return PFD_EINVAL;
                        scan_int(c.text.c_str(), &out->mla_u_size, 10);
                    } else if (c.name == "pitch") {
                        // every child of every "_" is read into the baseline: the last one wins
                        for (const Node& u : c.kids) {
                            if (u.name != "_") continue;
                            for (const Node& v : u.kids) {
                                if (!v.has_text) return PFD_EINVAL;
                                scan_f(v.text.c_str(), &out->baseline);
                            }
                        }
                    }
                }
            }
            out->has_mia = 1;
        } else if (g.name == "distortions") {
            for (const Node& e : g.kids) {
                double* dst = nullptr;
                int cnt = 0;
                if (e.name == "depth") { dst = out->distor_depth; cnt = 3; }
                else if (e.name == "radial") { dst = out->distor_radial; cnt = 3; }
                else if (e.name == "tangential") { dst = out->distor_tangential; cnt = 2; }
                if (!dst) continue;
                const Node* u = child(&e, 0);
                if (!u) return PFD_EINVAL;
                for (int i = 0; i < cnt; ++i) {
                    const char* t = text_of(child(u, (size_t)i));
                    if (!t) return PFD_EINVAL;
                    scan_lf(t, &dst[i]);
                }
            }
        }
    }
    return PFD_OK;
}

extern "C" pfd_status pfd_read_calib_xml(const char* text, pfd_mla_entry* out, int cap, int* n)
{
    if (!text || !n || cap < 0) return PFD_EINVAL;
    *n = 0;
    Node root;
    if (!Parser(text).document(root) || root.name != "Calib") return PFD_EINVAL;
    std::map<int, float> radius;                          // blur_type_radius_map
    std::map<std::pair<int, int>, pfd_mla_entry> lenses;  // m_MLA_info_map: key order (row, column)
    for (const Node& g : root.kids) {
        if (g.name == "BlurInfo") {
            for (const Node& e : g.kids) {
                if (e.name != "MLAType") continue;
                if (!e.has_text || !e.attr("id")) return PFD_EINVAL;
                float r = -1.0f;
                scan_f(e.text.c_str(), &r);
                int type = -1;
                scan_int(e.attr("id"), &type, 0);
                radius[type] = r;
            }
        } else if (g.name == "MLAInfo") {
            for (const Node& e : g.kids) {
                if (e.name != "MLA") continue;
                pfd_mla_entry m;
                m.col = -1; m.row = -1; m.cx = 0.0f; m.cy = 0.0f; m.type = -1; m.area = 0.0f;
                for (const Node& c : e.kids) {
                    // an empty element is skipped, as the reference's FirstChild() test
                    // does; one whose first child is an element has no text to read
                    if (!c.has_text) {
                        if (!c.kids.empty()) return PFD_EINVAL;
                        continue;
                    }
                    if (c.name == "key") scan_pair_i(c.text.c_str(), &m.row, &m.col);
                    else if (c.name == "center") scan_pair_f(c.text.c_str(), &m.cx, &m.cy);
                    else if (c.name == "MLAType") scan_int(c.text.c_str(), &m.type, 0);
                    else if (c.name == "aera") scan_f(c.text.c_str(), &m.area);
                }
                m.blur_radius = radius[m.type];                // operator[]: 0 for an unlisted type
                lenses[std::make_pair(m.row, m.col)] = m;
            }
        }
    }
    *n = (int)lenses.size();
    if (out) {
        if (*n > cap) return PFD_EINVAL;
        int i = 0;
        for (const auto& kv : lenses) out[i++] = kv.second;
    }
    return PFD_OK;
}

extern "C" pfd_status pfd_write_calib_xml(const pfd_mla_entry* lenses, const int* abandon, int n, char* buf,
                                          size_t buf_size, size_t* len)
{
    if (!len || n < 0 || (n > 0 && !lenses)) return PFD_EINVAL;
    std::map<std::pair<int, int>, int> order;             // key order, the map's iteration order
    for (int i = 0; i < n; ++i) order[std::make_pair(lenses[i].row, lenses[i].col)] = i;
    std::ostringstream o;                                  // default formatting: 6 significant digits
    o << "<Calib>\n    <BlurInfo>\n";
    for (int index = 0; index < 3; ++index) o << "        <MLAType id=\"" << index << "\">" << index << "</MLAType>\n";
    o << "    </BlurInfo>\n";
    std::ostringstream body;
    for (const auto& kv : order) {
        const int i = kv.second;
        if (abandon && abandon[i]) continue;
        const pfd_mla_entry& m = lenses[i];
        body << "        <MLA>\n";
        body << "            <key>" << m.row << "," << m.col << "</key>\n";
        body << "            <center>" << m.cx << "," << m.cy << "</center>\n";
        body << "            <MLAType>1</MLAType>\n";
        body << "            <aera>" << m.area << "</aera>\n";
        body << "        </MLA>\n";
    }
    const std::string b = body.str();
    if (b.empty()) o << "    <MLAInfo/>\n";
    else o << "    <MLAInfo>\n" << b << "    </MLAInfo>\n";
    o << "</Calib>\n";
    const std::string s = o.str();
    *len = s.size();
    if (buf) {
        if (buf_size <= s.size()) return PFD_EINVAL;
        std::memcpy(buf, s.c_str(), s.size() + 1);
    }
    return PFD_OK;
}
