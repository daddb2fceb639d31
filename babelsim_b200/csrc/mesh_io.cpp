// BABELSIM_MESH 3 reader (the reference's readMeshFile, src/io/mesh_reader.cpp:44-111),
// on the host: the file is read in one piece and tokenised in place, so a
// million-cell polyhedral mesh parses in well under a second, and the face
// rings land directly in the flat (offsets, ids) arrays the device geometry
// takes.  Rejections carry the reference's messages ("invalid BabelSim mesh
// file <path>: <what>"), and the token order and keyword checks are the
// reference's: header, vertices, faces (face <n> <owner> <neighbour> <patch>
// <ring...>), patches (patch <name> <kind>), end, nothing after.
#include "mesh_io.h"

#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>

namespace bsg {
namespace {

class Tokens {
public:
    Tokens(std::string path, std::string text) : path_(std::move(path)), text_(std::move(text)) {}

    [[noreturn]] void invalid(const std::string& message) const {
        fail(kArgument, "invalid BabelSim mesh file " + path_ + ": " + message);
    }
    // next whitespace-separated token; empty at the end of the file
    std::string word() {
        skip();
        const std::size_t b = pos_;
        while (pos_ < text_.size() && !space(text_[pos_])) ++pos_;
        return text_.substr(b, pos_ - b);
    }
    std::string word(const char* what) {
        std::string w = word();
        if (w.empty()) invalid(std::string("missing ") + what);
        return w;
    }
    long long integer(const char* what) {
        skip();
        if (pos_ >= text_.size()) invalid(std::string("missing ") + what);
        const char* s = text_.c_str() + pos_;
        char* end = nullptr;
        errno = 0;
        const long long v = std::strtoll(s, &end, 10);
        if (end == s || errno != 0 || (*end && !space(*end))) invalid(std::string("missing ") + what);
        pos_ += static_cast<std::size_t>(end - s);
        return v;
    }
    int index(const char* what) {
        const long long v = integer(what);
        if (v < std::numeric_limits<int>::min() || v > std::numeric_limits<int>::max())
            invalid(std::string("missing ") + what);
        return static_cast<int>(v);
    }
    int count(const char* what) {
        const int v = index(what);
        if (v <= 0 || v == std::numeric_limits<int>::max()) invalid(std::string(what) + " must be positive");
        return v;
    }
    double real(const char* what) {
        skip();
        if (pos_ >= text_.size()) invalid(std::string("missing ") + what);
        const char* s = text_.c_str() + pos_;
        char* end = nullptr;
        const double v = std::strtod(s, &end);
        if (end == s || (*end && !space(*end))) invalid(std::string("missing ") + what);
        pos_ += static_cast<std::size_t>(end - s);
        return v;
    }

private:
    static bool space(char c) { return c == ' ' || c == '\n' || c == '\t' || c == '\r' || c == '\v' || c == '\f'; }
    void skip() {
        while (pos_ < text_.size() && space(text_[pos_])) ++pos_;
    }
    std::string path_, text_;
    std::size_t pos_ = 0;
};

int patchKind(const std::string& name, const Tokens& t) {
    if (name == "generic") return 0;
    if (name == "wall") return 1;
    if (name == "inlet") return 2;
    if (name == "outlet") return 3;
    if (name == "symmetry" || name == "mirror") return 4;
    if (name == "processor") return 5;
    t.invalid("unknown patch kind " + name);
}

}  // namespace

PolyFile readPolyFile(const std::string& path) {
    std::FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) fail(kArgument, "cannot open BabelSim mesh file: " + path);
    std::string text;
    char buf[1 << 16];
    std::size_t got;
    while ((got = std::fread(buf, 1, sizeof(buf), f)) > 0) text.append(buf, got);
    std::fclose(f);
    Tokens t(path, std::move(text));
    PolyFile m;
    const std::string magic = t.word("file header");
    const int version = t.index("format version");
    if (magic != "BABELSIM_MESH" || version != 3) t.invalid("only BABELSIM_MESH version 3 is supported");
    if (t.word("vertices keyword") != "vertices") t.invalid("expected vertices");
    const int nv = t.count("vertex count");
    m.vertices.resize(3 * static_cast<std::size_t>(nv));
    for (int v = 0; v < nv; ++v) {
        const double x = t.real("vertex x"), y = t.real("vertex y"), z = t.real("vertex z");
        if (!std::isfinite(x) || !std::isfinite(y) || !std::isfinite(z)) t.invalid("vertex must be finite");
        m.vertices[3 * static_cast<std::size_t>(v)] = x;
        m.vertices[3 * static_cast<std::size_t>(v) + 1] = y;
        m.vertices[3 * static_cast<std::size_t>(v) + 2] = z;
    }
    if (t.word("faces keyword") != "faces") t.invalid("expected faces");
    const int nf = t.count("face count");
    m.offsets.reserve(static_cast<std::size_t>(nf) + 1);
    m.offsets.push_back(0);
    m.owner.resize(nf);
    m.neighbour.resize(nf);
    m.patch.resize(nf);
    for (int face = 0; face < nf; ++face) {
        if (t.word("face keyword") != "face") t.invalid("expected face");
        const int k = t.count("face vertex count");
        m.owner[face] = t.index("face owner");
        m.neighbour[face] = t.index("face neighbour");
        m.patch[face] = t.index("face patch");
        for (int q = 0; q < k; ++q) m.ids.push_back(t.index("face vertex index"));
        m.offsets.push_back(static_cast<int>(m.ids.size()));
    }
    if (t.word("patches keyword") != "patches") t.invalid("expected patches");
    const int np = t.count("patch count");
    for (int p = 0; p < np; ++p) {
        if (t.word("patch keyword") != "patch") t.invalid("expected patch");
        const std::string name = t.word("patch name");
        const int kind = patchKind(t.word("patch kind"), t);
        if (name.empty()) t.invalid("patch name must not be empty");
        m.patch_names.push_back(name);
        m.patch_kinds.push_back(kind);
    }
    if (t.word("end marker") != "end") t.invalid("expected end");
    const std::string trailing = t.word();
    if (!trailing.empty()) t.invalid("unexpected trailing token " + trailing);
    // Mesh::polyhedral's checks, with the reader's prefix as readMeshFile adds it
    try {
        m.n_cells = validatePolyhedralTopology(nv, nf, m.offsets.data(), m.ids.data(), m.owner.data(),
                                               m.neighbour.data(), m.patch.data(), np);
    } catch (const Error& e) {
        t.invalid(e.what());
    }
    return m;
}

}  // namespace bsg
