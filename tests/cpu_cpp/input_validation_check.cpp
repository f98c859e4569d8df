// Input validation of the drop-in host classes, without a GPU: malformed XML
// must raise dvm::XMLParseException (src/XmlHandler.cpp:25-50 throws it for a
// missing or invalid option; main turns it into rc = 1, src/main.cpp:103-112),
// well-formed XML with comments, CDATA, entities and character references must
// load, and a body file that is not a usable closed contour must raise
// dvm::FileIOException from VortexSheet's constructor before any device call
// (the reference throws FileIOException for an unreadable domain file,
// src/VortexSheet.cpp:62-64).  Built and run by tests/test_input_validation.py;
// prints "ok" or the first failure.
#include <cmath>
#include <cstdio>
#include <fstream>
#include <functional>
#include <string>

#include "Exceptions.hpp"
#include "VortexSheet.hpp"
#include "XmlHandler.hpp"

static std::string g_dir;
static int g_fail = 0;

static std::string write(const std::string& name, const std::string& text) {
    const std::string p = g_dir + "/" + name;
    std::ofstream f(p);
    f << text;
    return p;
}

template <class E>
static void expect_throw(const char* what, const std::function<void()>& fn,
                         const char* must_contain = nullptr) {
    try {
        fn();
    } catch (const E& e) {
        if (must_contain && std::string(e.what()).find(must_contain) == std::string::npos) {
            std::printf("%s: message '%s' lacks '%s'\n", what, e.what(), must_contain);
            g_fail = 1;
        }
        return;
    } catch (const std::exception& e) {
        std::printf("%s: wrong exception type: %s\n", what, e.what());
        g_fail = 1;
        return;
    }
    std::printf("%s: no exception\n", what);
    g_fail = 1;
}

static std::string case_xml(const std::string& body, const std::string& extra_constants = "") {
    return "<?xml version=\"1.0\"?>\n<DVMpp>\n"
           "  <algorithms><surface_crossing string=\"REFLECT\" /></algorithms>\n"
           "  <constants>\n"
           "    <density val=\"1\" /><nu val=\"0.001\" /><max_NumPanelVort val=\"3\" />\n"
           "    <cutoff_exp val=\"0.675\" /><seed val=\"1\" />" + extra_constants + "\n"
           "  </constants>\n"
           "  <io><input_dir string=\"" + g_dir + "/\" /><output_dir string=\"" + g_dir +
           "/\" /><domain_file string=\"" + body + "\" /></io>\n"
           "  <flow><ux val=\"1\" /><uz val=\"0\" /></flow>\n"
           "  <probe><x val=\"2\" /><z val=\"0\" /></probe>\n"
           "  <time><scheme string=\"euler\" /><dt val=\"0.005\" /><steps val=\"10\" /></time>\n"
           "</DVMpp>\n";
}

static std::string circle_text(int np, bool close = true, int repeat = -1, bool nan = false) {
    std::string t;
    const int npts = close ? np + 1 : np;
    for (int i = 0; i < npts; ++i) {
        const int k = (i == repeat) ? i - 1 : i % np;
        double x = 0.5 * std::cos(2.0 * M_PI * k / np), z = 0.5 * std::sin(2.0 * M_PI * k / np);
        if (nan && i == 3) x = std::nan("");
        char b[96];
        std::snprintf(b, sizeof b, "%.17g %.17g\n", x, z);
        t += b;
    }
    return t;
}

int main(int argc, char** argv) {
    g_dir = argc > 1 ? argv[1] : ".";

    // ---- well-formed XML with comments, CDATA, entities, character references
    {
        const std::string p = write(
            "ok.xml",
            "<?xml version=\"1.0\"?>\n<!DOCTYPE DVMpp>\n<!-- leading comment -->\n<DVMpp>\n"
            "  <io><input_dir string=\"a&lt;b&amp;c&#65;&#x42;\" /><!-- c <io> -->\n"
            "  <![CDATA[ <not> an element ]]>\n"
            "  <output_dir string='single &quot;quoted&quot;' /></io>\n"
            "  <constants><nu val=\"0.25\"/></constants>\n"
            "</DVMpp>\n");
        XmlHandler x(p);
        if (x.getStringAttribute("io", "input_dir") != "a<b&cAB") {
            std::printf("entities: got '%s'\n", x.getStringAttribute("io", "input_dir").c_str());
            g_fail = 1;
        }
        if (x.getStringAttribute("io", "output_dir") != "single \"quoted\"") {
            std::printf("quotes: got '%s'\n", x.getStringAttribute("io", "output_dir").c_str());
            g_fail = 1;
        }
        if (x.getValueAttribute("constants", "nu") != 0.25) {
            std::printf("nu: got %g\n", x.getValueAttribute("constants", "nu"));
            g_fail = 1;
        }
        // a missing option and a value outside the allowed list (reference semantics)
        expect_throw<dvm::XMLParseException>("missing parameter",
                                             [&] { x.getValueAttribute("constants", "density"); },
                                             "missing");
        expect_throw<dvm::XMLParseException>("unmapped option",
                                             [&] { x.getValueAttribute("io", "nonsense"); });
    }
    {
        const std::string p = write("badopt.xml",
                                    "<DVMpp><algorithms><surface_crossing string=\"BOUNCE\"/>"
                                    "</algorithms><constants><nu val=\"-1\"/></constants></DVMpp>");
        XmlHandler x(p);
        expect_throw<dvm::XMLParseException>(
            "invalid string option", [&] { x.getStringAttribute("algorithms", "surface_crossing"); },
            "Valid options");
        expect_throw<dvm::XMLParseException>("non-positive value",
                                             [&] { x.getValueAttribute("constants", "nu"); });
    }

    // ---- malformed XML: every one must be an XMLParseException from the constructor
    const char* bad[][2] = {
        {"unterminated element", "<DVMpp><io><input_dir string=\"a\" /></io>"},
        {"mismatched close tag", "<DVMpp><io></constants></DVMpp>"},
        {"unquoted attribute", "<DVMpp><io><input_dir string=a /></io></DVMpp>"},
        {"unterminated attribute", "<DVMpp><io><input_dir string=\"a /></io></DVMpp>"},
        {"attribute without value", "<DVMpp><io><input_dir string /></io></DVMpp>"},
        {"unterminated comment", "<DVMpp><!-- never closed </DVMpp>"},
        {"unterminated CDATA", "<DVMpp><![CDATA[ never closed </DVMpp>"},
        {"text outside the root", "hello <DVMpp></DVMpp>"},
        {"empty document", ""},
        {"only a declaration", "<?xml version=\"1.0\"?>\n"},
        {"bad character reference", "<DVMpp><io><input_dir string=\"&#xZZ;\" /></io></DVMpp>"},
        {"element name missing", "<DVMpp>< /></DVMpp>"},
    };
    for (const auto& b : bad) {
        const std::string p = write("bad.xml", b[1]);
        expect_throw<dvm::XMLParseException>(b[0], [&] { XmlHandler x(p); }, "Cannot load XML");
    }
    expect_throw<dvm::XMLParseException>("missing file",
                                         [&] { XmlHandler x(g_dir + "/does_not_exist.xml"); },
                                         "not found");

    // ---- body contours that are not a usable closed polygon
    struct Body {
        const char* what;
        std::string text;
        const char* msg;
    } bodies[] = {
        {"open contour", circle_text(32, false), "not closed"},
        {"repeated point (zero-length panel)", circle_text(32, true, 5), "zero length"},
        {"NaN coordinate", circle_text(32, true, -1, true), "not finite"},
        {"two panels", "0 0\n1 0\n0 0\n", "at least 3 panels"},
        {"one column", "0.5\n0.25\n", "Cannot read"},
        {"three columns", "0 0 0\n1 0 0\n0 1 0\n0 0 0\n", "Cannot read"},
        {"text", "zero zero\n", "Cannot read"},
    };
    for (const auto& b : bodies) {
        write("body.txt", b.text);
        const std::string p = write("case.xml", case_xml("body.txt"));
        XmlHandler x(p);
        expect_throw<dvm::FileIOException>(b.what, [&] { VortexSheet s(x, "t"); }, b.msg);
    }
    {
        const std::string p = write("case.xml", case_xml("missing_body.txt"));
        XmlHandler x(p);
        expect_throw<dvm::FileIOException>("missing body file", [&] { VortexSheet s(x, "t"); },
                                           "Cannot read");
    }
    if (!g_fail) std::printf("ok\n");
    return g_fail;
}
