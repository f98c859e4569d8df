#include "XmlHandler.hpp"

#include <cctype>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <sstream>
#include <stdexcept>

#include "Exceptions.hpp"

namespace dvm {

const XmlNode* XmlNode::child(const std::string& n) const {
    for (const auto& c : children)
        if (c->name == n) return c.get();
    return nullptr;
}

const std::string* XmlNode::attr(const std::string& n) const {
    for (const auto& a : attrs)
        if (a.first == n) return &a.second;
    return nullptr;
}

namespace {

struct Reader {
    const std::string& s;
    size_t i = 0;
    explicit Reader(const std::string& t) : s(t) {}
    [[noreturn]] void error(const std::string& what) const {
        throw std::runtime_error(what + " at offset " + std::to_string(i));
    }
    bool starts(const char* p) const { return s.compare(i, std::char_traits<char>::length(p), p) == 0; }
    void skip_ws() {
        while (i < s.size() && std::isspace((unsigned char)s[i])) ++i;
    }
    void skip_past(const char* end) {
        const size_t k = s.find(end, i);
        if (k == std::string::npos) error(std::string("unterminated construct, expected ") + end);
        i = k + std::char_traits<char>::length(end);
    }
    // comments, processing instructions and declarations between elements
    void skip_misc() {
        for (;;) {
            skip_ws();
            if (starts("<!--")) skip_past("-->");
            else if (starts("<![CDATA[")) skip_past("]]>");  // character data: ignored
            else if (starts("<?")) skip_past("?>");
            else if (starts("<!")) skip_past(">");
            else return;
        }
    }
    std::string name() {
        const size_t b = i;
        while (i < s.size() && (std::isalnum((unsigned char)s[i]) || s[i] == '_' || s[i] == '-' ||
                                s[i] == '.' || s[i] == ':'))
            ++i;
        if (i == b) error("expected a name");
        return s.substr(b, i - b);
    }
    static void append_utf8(std::string& o, unsigned long cp) {
        if (cp < 0x80) {
            o += (char)cp;
        } else if (cp < 0x800) {
            o += (char)(0xC0 | (cp >> 6));
            o += (char)(0x80 | (cp & 0x3F));
        } else if (cp < 0x10000) {
            o += (char)(0xE0 | (cp >> 12));
            o += (char)(0x80 | ((cp >> 6) & 0x3F));
            o += (char)(0x80 | (cp & 0x3F));
        } else {
            o += (char)(0xF0 | (cp >> 18));
            o += (char)(0x80 | ((cp >> 12) & 0x3F));
            o += (char)(0x80 | ((cp >> 6) & 0x3F));
            o += (char)(0x80 | (cp & 0x3F));
        }
    }
    static std::string unescape(const std::string& v) {
        std::string o;
        for (size_t k = 0; k < v.size(); ++k) {
            if (v[k] != '&') {
                o += v[k];
                continue;
            }
            const size_t e = v.find(';', k);
            const std::string ent = e == std::string::npos ? "" : v.substr(k + 1, e - k - 1);
            if (ent == "lt") o += '<';
            else if (ent == "gt") o += '>';
            else if (ent == "amp") o += '&';
            else if (ent == "quot") o += '"';
            else if (ent == "apos") o += '\'';
            else if (ent.size() > 1 && ent[0] == '#') {  // &#65; or &#x41;
                const bool hex = ent[1] == 'x' || ent[1] == 'X';
                char* end = nullptr;
                const unsigned long cp = std::strtoul(ent.c_str() + (hex ? 2 : 1), &end, hex ? 16 : 10);
                if (!end || *end != '\0' || cp == 0 || cp > 0x10FFFF)
                    throw std::runtime_error("bad character reference &" + ent + ";");
                append_utf8(o, cp);
            } else {
                o += v[k];
                continue;
            }
            k = e;
        }
        return o;
    }
    std::unique_ptr<XmlNode> element() {
        if (i >= s.size() || s[i] != '<') error("expected '<'");
        ++i;
        auto n = std::make_unique<XmlNode>();
        n->name = name();
        for (;;) {
            skip_ws();
            if (starts("/>")) {
                i += 2;
                return n;
            }
            if (i < s.size() && s[i] == '>') {
                ++i;
                break;
            }
            std::string an = name();
            skip_ws();
            if (i >= s.size() || s[i] != '=') error("expected '=' after attribute " + an);
            ++i;
            skip_ws();
            if (i >= s.size() || (s[i] != '"' && s[i] != '\'')) error("expected a quoted value");
            const char q = s[i++];
            const size_t e = s.find(q, i);
            if (e == std::string::npos) error("unterminated attribute value");
            n->attrs.emplace_back(an, unescape(s.substr(i, e - i)));
            i = e + 1;
        }
        for (;;) {  // content: child elements; character data is ignored
            skip_misc();
            if (i >= s.size()) error("unterminated element <" + n->name + ">");
            if (starts("</")) {
                i += 2;
                const std::string closing = name();
                if (closing != n->name) error("mismatched </" + closing + "> for <" + n->name + ">");
                skip_ws();
                if (i >= s.size() || s[i] != '>') error("expected '>'");
                ++i;
                return n;
            }
            if (s[i] == '<') {
                n->children.push_back(element());
            } else {
                while (i < s.size() && s[i] != '<') ++i;
            }
        }
    }
};

void write_node(std::ostringstream& o, const XmlNode& n, int depth) {
    const std::string pad(2 * depth, ' ');
    o << pad << '<' << n.name;
    for (const auto& a : n.attrs) o << ' ' << a.first << "=\"" << a.second << '"';
    if (n.children.empty()) {
        o << " />\n";
        return;
    }
    o << ">\n";
    for (const auto& c : n.children) write_node(o, *c, depth + 1);
    o << pad << "</" << n.name << ">\n";
}

}  // namespace

std::unique_ptr<XmlNode> parse_xml(const std::string& text) {
    Reader r(text);
    auto root = std::make_unique<XmlNode>();
    for (;;) {
        r.skip_misc();
        if (r.i >= text.size()) break;
        root->children.push_back(r.element());
    }
    if (root->children.empty()) throw std::runtime_error("no document element");
    return root;
}

std::string write_xml(const XmlNode& root) {
    std::ostringstream o;
    o << "<?xml version=\"1.0\"?>\n";
    for (const auto& c : root.children) write_node(o, *c, 0);
    return o.str();
}

}  // namespace dvm

// ---------------------------------------------------------------------------
XmlHandler::XmlHandler() { buildOptionMap(); }

XmlHandler::XmlHandler(std::string xml_file) {
    std::ifstream f(xml_file, std::ios::binary);
    if (!f) throw dvm::XMLParseException::cannotLoad(xml_file, "File was not found");
    std::stringstream ss;
    ss << f.rdbuf();
    try {
        m_doc = dvm::parse_xml(ss.str());
    } catch (const std::exception& e) {
        throw dvm::XMLParseException::cannotLoad(xml_file, e.what());
    }
    std::cout << "Loaded xml input: " << xml_file << "\n";
    buildOptionMap();
}

static std::unique_ptr<dvm::XmlNode> clone(const dvm::XmlNode& n) {
    auto c = std::make_unique<dvm::XmlNode>();
    c->name = n.name;
    c->attrs = n.attrs;
    for (const auto& ch : n.children) c->children.push_back(clone(*ch));
    return c;
}

XmlHandler::XmlHandler(const XmlHandler& o) : m_option_map(o.m_option_map) {
    if (o.m_doc) m_doc = clone(*o.m_doc);
}

XmlHandler& XmlHandler::operator=(const XmlHandler& o) {
    if (this != &o) {
        m_doc = o.m_doc ? clone(*o.m_doc) : nullptr;
        m_option_map = o.m_option_map;
    }
    return *this;
}

std::string XmlHandler::form_key(const char* level, const char* parameter) const {
    return std::string(level) + "_" + parameter;
}

bool XmlHandler::has(const char* level, const char* parameter) const {
    if (!m_doc) return false;
    const dvm::XmlNode* top = m_doc->child("DVMpp");
    const dvm::XmlNode* l = top ? top->child(level) : nullptr;
    return l && l->child(parameter);
}

const dvm::XmlNode& XmlHandler::getNode(const char* level, const char* parameter) const {
    const dvm::XmlNode* top = m_doc ? m_doc->child("DVMpp") : nullptr;
    const dvm::XmlNode* l = top ? top->child(level) : nullptr;
    const dvm::XmlNode* p = l ? l->child(parameter) : nullptr;
    const auto it = m_option_map.find(form_key(level, parameter));
    if (!p) {
        std::ostringstream err;
        if (it != m_option_map.end()) {
            err << "xml error: <" << level << "><" << parameter << "> missing.\nAttribute: "
                << it->second.attr << "\nInfo: " << it->second.info
                << "\nOptions: " << it->second.reqs;
        } else {
            err << "xml error: Are you trying to add an option without updating "
                   "XmlHandler::m_option_map?\nRequested option: <"
                << level << "><" << parameter << ">";
        }
        throw dvm::XMLParseException(err.str());
    }
    if (it == m_option_map.end())
        throw dvm::XMLParseException("<" + std::string(level) + "><" + parameter +
                                     "> not found in the option map.");
    return *p;
}

void XmlHandler::check_string(const char* level, const char* parameter, std::string& attr) const {
    const std::string& req = m_option_map.find(form_key(level, parameter))->second.reqs;
    if (req == "none") return;
    if (req.find(attr) == std::string::npos)  // substring test, as the reference does
        throw dvm::XMLParseException::invalidOption(level, parameter, req);
}

void XmlHandler::check_value(const char* level, const char* parameter, double attr) const {
    const std::string& req = m_option_map.find(form_key(level, parameter))->second.reqs;
    if (req == "none") return;
    if (req == ">0") {
        if (attr <= 0) throw dvm::XMLParseException::invalidOption(level, parameter, req);
        return;
    }
    throw dvm::XMLParseException::invalidOption(level, parameter, req);
}

std::string XmlHandler::getStringAttribute(const char* level, const char* parameter,
                                           bool checksep) const {
    const std::string* a = getNode(level, parameter).attr("string");
    std::string v = a ? *a : std::string();
    check_string(level, parameter, v);
    if (checksep && (v.empty() || v.back() != '/')) v += '/';
    return v;
}

std::vector<double> XmlHandler::getList(const char* level, const char* parameter) const {
    const std::string* a = getNode(level, parameter).attr("string");
    std::string v = a ? *a : std::string();
    check_string(level, parameter, v);
    std::vector<double> out;
    std::istringstream s(v);
    double d;
    while (s >> d) {
        out.push_back(d);
        if (s.peek() == ' ' || s.peek() == ',') s.ignore();
    }
    return out;
}

double XmlHandler::getValueAttribute(const char* level, const char* parameter) const {
    const std::string* a = getNode(level, parameter).attr("val");
    const double v = a ? std::strtod(a->c_str(), nullptr) : 0.0;
    check_value(level, parameter, v);
    return v;
}

int XmlHandler::getIntAttribute(const char* level, const char* parameter) const {
    const std::string* a = getNode(level, parameter).attr("val");
    return a ? (int)std::strtol(a->c_str(), nullptr, 10) : 0;
}

bool XmlHandler::getBoolAttribute(const char* level, const char* parameter) const {
    const std::string* a = getNode(level, parameter).attr("string");
    if (!a || a->empty()) return false;
    const char c = (*a)[0];
    return c == '1' || c == 't' || c == 'T' || c == 'y' || c == 'Y';
}

void XmlHandler::save(std::string filename) const {
    std::ofstream f(filename);
    if (m_doc) f << dvm::write_xml(*m_doc);
}

void XmlHandler::writeExample(std::string file) const {
    dvm::XmlNode root;
    auto top = std::make_unique<dvm::XmlNode>();
    top->name = "DVMpp";
    for (const auto& e : m_option_map) {
        const opts& o = e.second;
        dvm::XmlNode* lvl = nullptr;
        for (auto& c : top->children)
            if (c->name == o.level) lvl = c.get();
        if (!lvl) {
            top->children.push_back(std::make_unique<dvm::XmlNode>());
            lvl = top->children.back().get();
            lvl->name = o.level;
        }
        auto p = std::make_unique<dvm::XmlNode>();
        p->name = o.parameter;
        p->attrs.emplace_back(o.attr, o.info + ". Options: " + o.reqs);
        lvl->children.push_back(std::move(p));
    }
    root.children.push_back(std::move(top));
    if (file == "-") {
        std::cout << dvm::write_xml(root);
    } else {
        std::cout << "Saving example xml to " << file << std::endl;
        std::ofstream f(file);
        f << dvm::write_xml(root);
    }
}

void XmlHandler::buildOptionMap() {
    // (level, parameter, attribute, description, allowed values) -- the
    // reference's keys (src/XmlHandler.cpp:162-202) plus the GPU choices.
    const opts table[] = {
        {"algorithms", "surface_crossing", "string", "surface-crossing algorithm", "DELETE ABSORB REFLECT"},
        {"algorithms", "velocity_kernel", "string", "velocity computation kernel", "direct fmm cuda cuda64"},
        {"algorithms", "diffusion_rng", "string", "random walk source", "inject philox"},
        {"algorithms", "fmm_expansion_order", "val", "FMM expansion order", ">0"},
        {"algorithms", "fmm_theta", "val", "FMM opening angle criterion", "none"},
        {"algorithms", "merge_threshold", "val", "vortex merge threshold (0=disabled)", "none"},
        {"algorithms", "merge_frequency", "val", "merge every N steps (0=disabled)", "none"},
        {"constants", "density", "val", "specific gravity of fluid", ">0"},
        {"constants", "nu", "val", "kinematic viscosity [m^2 / s]", ">0"},
        {"constants", "max_NumPanelVort", "val", "maximum number of panel vortices", ">0"},
        {"constants", "cutoff_exp", "val", "cutoff exp", "none"},
        {"constants", "seed", "val", "seed for rng. <0 random, >=0 seed", "none"},
        {"io", "input_dir", "string", "input directory", "none"},
        {"io", "output_dir", "string", "output directory", "none"},
        {"io", "domain_file", "string", "body geometry file", "none"},
        {"flow", "ux", "val", "flow in the x-direction", "none"},
        {"flow", "uz", "val", "flow in the z-direction", "none"},
        {"probe", "x", "val", "x-coordinate of the probe", "none"},
        {"probe", "z", "val", "z-coordinate of the probe", "none"},
        {"time", "scheme", "string", "time-stepping scheme", "euler RK3"},
        {"time", "dt", "val", "time step [s]", ">0"},
        {"time", "steps", "val", "total number of timesteps", ">0"},
        {"remesh", "frequency", "val", "remesh every N steps (0=disabled)", "none"},
        {"remesh", "xmin", "val", "mesh x-direction minimum bound", "none"},
        {"remesh", "xmax", "val", "mesh x-direction maximum bound", "none"},
        {"remesh", "zmin", "val", "mesh z-direction minimum bound", "none"},
        {"remesh", "zmax", "val", "mesh z-direction maximum bound", "none"},
        {"remesh", "dx", "val", "mesh spacing in x-direction", ">0"},
        {"remesh", "dz", "val", "mesh spacing in z-direction", ">0"},
        {"remesh", "kernel", "string", "interpolation kernel", "M4prime gaussian M6"},
        {"remesh", "sigma", "val", "core size for new particles", ">0"},
        {"remesh", "circ_threshold", "val", "minimum circulation for particle creation", "none"},
    };
    for (const opts& o : table)
        m_option_map.emplace(o.level + "_" + o.parameter, o);
}
