// The gmsh .msh reader behind cfg_mesh_read_gmsh, the device path's
// counterpart of GmshMesh::fromFile (src/3d/src/mesh/gmshMesh.cpp:534-776).
//
// Supported input, as the reference accepts it: ASCII files of format 2.2
// or 4.x with first-order tetrahedra, hexahedra and prisms.  Boundary faces
// take the name of the physical group of the surface element on them (for a
// quad face, also that of a triangle a triangulated surface split it into),
// else the bounding-box plane they lie on (meshFromCells).
//
// How it reads.  The file is loaded in one piece and split into lines; the
// lines whose first token starts with '$' are the only ones that can open or
// close a section, so locating a section walks those alone.  A section's
// lines are tokenised on the host's threads into one flat array of string
// views, and its readers then move a cursor over the resulting rows.  Bulk
// rows (node coordinates, element connectivity) are decoded in parallel
// chunks; when several rows are bad, the error reported is the first one in
// file order, as a serial reader would report it.  Elements are read in two
// passes: the layout pass validates every row's shape and collects where
// its node columns start; the decode pass then maps node tags to points and
// checks each element's nodes.  Layout errors therefore come before node
// errors, as in the reference's reader.
//
// Messages keep the reference's wording (kMessages below) so a caller's
// error handling sees the same text from either reader.
#include <algorithm>
#include <array>
#include <cctype>
#include <cerrno>
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <initializer_list>
#include <map>
#include <numeric>
#include <string>
#include <string_view>
#include <vector>

#include "cfg_internal.h"

namespace cfg
{
namespace
{

// ---------------------------------------------------------------------------
// messages
// ---------------------------------------------------------------------------

enum class Msg
{
    CannotOpen, CannotRead, MissingSection, Unterminated, RanOut, NotAnInteger, NotANumber,
    BadFormatRow, BinaryFile, UnsupportedVersion,
    BadGroupRow, UnnamedGroup,
    EmptyNodes, BadNodeRow, BadCoordinates, BadNodesHeader, BadNodeBlockHeader, NodeCountMismatch,
    NodeTagCountMismatch, DuplicateNodeTag,
    BadEntityNameRow, BadEntitiesHeader, BadSurfaceEntity,
    EmptyElements, BadElementRow, NotFirstOrder, ShortElementRow, BadElementsHeader, BadElementBlockHeader,
    ElementWidth, ElementWidthChanged, ElementCountMismatch, UnknownNode, RepeatedNode, Pyramid,
    NoVolumes,
};

/// The text of each message; every '@' is replaced by the next argument.
constexpr std::pair<Msg, const char*> kMessages[] = {
    {Msg::CannotOpen, "gmsh: cannot open @"},
    {Msg::CannotRead, "gmsh: cannot read @"},
    {Msg::MissingSection, "gmsh: @ has no @ section"},
    {Msg::Unterminated, "gmsh: section @ in @ is not terminated"},
    {Msg::RanOut, "gmsh: truncated file: @ ends after @ rows"},
    {Msg::NotAnInteger, "gmsh: expected an integer but found '@' in @"},
    {Msg::NotANumber, "gmsh: expected a number but found '@' in @"},
    {Msg::BadFormatRow, "gmsh: malformed $MeshFormat in @"},
    {Msg::BinaryFile, "gmsh: @ is a binary .msh; write it with Mesh.Binary = 0"},
    {Msg::UnsupportedVersion, "gmsh: format '@' is not supported (ASCII 2.2 and 4.1 are)"},
    {Msg::BadGroupRow, "gmsh: malformed $PhysicalNames entry"},
    {Msg::UnnamedGroup, "gmsh: physical group @ has no name"},
    {Msg::EmptyNodes, "gmsh: @ has an empty $Nodes section"},
    {Msg::BadNodeRow, "gmsh: malformed node line in @"},
    {Msg::BadCoordinates, "gmsh: malformed node coordinate in $Nodes"},
    {Msg::BadNodesHeader, "gmsh: malformed $Nodes header in @"},
    {Msg::BadNodeBlockHeader, "gmsh: malformed $Nodes block header in @"},
    {Msg::NodeCountMismatch, "gmsh: $Nodes declares @ nodes, @ were read from @ (unsupported node layout?)"},
    {Msg::NodeTagCountMismatch, "gmsh: a $Nodes block in @ lists @ tags for @ nodes"},
    {Msg::DuplicateNodeTag, "gmsh: duplicate node tag @ in @"},
    {Msg::BadEntityNameRow, "gmsh: malformed $EntityNames entry"},
    {Msg::BadEntitiesHeader, "gmsh: malformed $Entities header"},
    {Msg::BadSurfaceEntity, "gmsh: malformed $Entities surface line"},
    {Msg::EmptyElements, "gmsh: @ has an empty $Elements section"},
    {Msg::BadElementRow, "gmsh: malformed element line in @"},
    {Msg::NotFirstOrder, "gmsh: element type @ in @ is not a first-order element; mesh with Linear order"},
    {Msg::ShortElementRow, "gmsh: truncated element line in @"},
    {Msg::BadElementsHeader, "gmsh: malformed $Elements header in @"},
    {Msg::BadElementBlockHeader, "gmsh: malformed $Elements block header in @"},
    {Msg::ElementWidth, "gmsh: element line with @ entries, expected @ or @"},
    {Msg::ElementWidthChanged, "gmsh: inconsistent element line width in @"},
    {Msg::ElementCountMismatch,
     "gmsh: $Elements declares @ elements, @ were read from @ (unsupported element layout?)"},
    {Msg::UnknownNode, "gmsh: an element refers to node @, which $Nodes does not define"},
    {Msg::RepeatedNode, "gmsh: element @ repeats a node"},
    {Msg::Pyramid, "gmsh: pyramid elements are not supported"},
    {Msg::NoVolumes, "gmsh: @ has no volume elements"},
};

std::string str(long v) { return std::to_string(v); }

[[noreturn]] void raise(Msg id, std::initializer_list<std::string> args = {})
{
    const char* text = "gmsh: error";
    for (const auto& m : kMessages)
        if (m.first == id) text = m.second;
    std::string out;
    auto arg = args.begin();
    for (const char* c = text; *c; ++c)
    {
        if (*c == '@' && arg != args.end()) out += *arg++;
        else out += *c;
    }
    fail(CFG_EMESH, out);
}

// ---------------------------------------------------------------------------
// numbers
// ---------------------------------------------------------------------------

/// std::stol's reading of a token (leading sign, digits up to the first
/// other character), without a copy when the token is just the number.
long parseInt(std::string_view tok, const char* context)
{
    const char* b = tok.data();
    const char* e = b + tok.size();
    if (b < e && *b == '+') ++b;
    long v = 0;
    const auto r = std::from_chars(b, e, v);
    if (r.ec == std::errc() && r.ptr == e) return v;
    const std::string s(tok);
    char* stop = nullptr;
    errno = 0;
    v = std::strtol(s.c_str(), &stop, 10);
    if (stop == s.c_str() || errno == ERANGE) raise(Msg::NotAnInteger, {s, context});
    return v;
}

/// std::stod's reading of a token; from_chars rounds as strtod does.
double parseReal(std::string_view tok, const char* context)
{
    const char* b = tok.data();
    const char* e = b + tok.size();
    if (b < e && *b == '+') ++b;
    double v = 0;
    const auto r = std::from_chars(b, e, v);
    if (r.ec == std::errc() && r.ptr == e) return v;
    const std::string s(tok);
    char* stop = nullptr;
    errno = 0;
    v = std::strtod(s.c_str(), &stop);
    if (stop == s.c_str() || errno == ERANGE) raise(Msg::NotANumber, {s, context});
    return v;
}

/// a token written without a fraction or exponent (a node-tag line)
bool looksIntegral(std::string_view tok) { return tok.find_first_of(".eE") == std::string_view::npos; }

// ---------------------------------------------------------------------------
// sections as rows of tokens
// ---------------------------------------------------------------------------

/// One row: a span of a section's token array.
struct Row
{
    const std::string_view* tok = nullptr;
    size_t n = 0;
    const std::string_view& operator[](size_t i) const { return tok[i]; }
};

/// The non-empty rows between $Name and $EndName.
struct SectionRows
{
    std::vector<std::string_view> tokens;
    std::vector<size_t> rowEnd;  // token index one past each row's last token
    std::string label;           // "$Name in <path>", for the ran-out message

    size_t rows() const { return rowEnd.size(); }
    Row row(size_t i) const
    {
        const size_t b = i ? rowEnd[i - 1] : 0;
        return Row{tokens.data() + b, rowEnd[i] - b};
    }
};

/// A read position in a section.  Asking for a row past the last one is
/// the truncated-file error.
class Cursor
{
public:
    explicit Cursor(const SectionRows& s) : s_(s) {}
    size_t left() const { return s_.rows() - at_; }
    Row next()
    {
        if (at_ >= s_.rows()) raise(Msg::RanOut, {s_.label, std::to_string(s_.rows())});
        return s_.row(at_++);
    }
    /// the row k places ahead (k < left()), not consumed
    Row ahead(size_t k) const { return s_.row(at_ + k); }
    void skip(size_t k) { at_ += k; }
    /// consumes the next row when it is one integral token (a node tag)
    bool nextTag(long& tag)
    {
        if (at_ >= s_.rows()) return false;
        const Row r = s_.row(at_);
        if (r.n != 1 || !looksIntegral(r[0])) return false;
        tag = parseInt(r[0], s_.label.c_str());
        ++at_;
        return true;
    }

private:
    const SectionRows& s_;
    size_t at_ = 0;
};

bool isBlank(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\v' || c == '\f'; }

/// The file's text with its line index.
class MshText
{
public:
    explicit MshText(const std::string& path) : path_(path)
    {
        std::FILE* fp = std::fopen(path.c_str(), "rb");
        if (!fp) raise(Msg::CannotOpen, {path});
        std::fseek(fp, 0, SEEK_END);
        const long size = std::ftell(fp);
        std::fseek(fp, 0, SEEK_SET);
        text_.resize(static_cast<size_t>(std::max(size, 0L)));
        const size_t got = size > 0 ? std::fread(&text_[0], 1, text_.size(), fp) : 0;
        std::fclose(fp);
        if (got != text_.size()) raise(Msg::CannotRead, {path});
        // lines end at '\n'; the last one may lack it
        const char* t = text_.data();
        const size_t n = text_.size();
        for (size_t b = 0; b < n;)
        {
            const void* nl = std::memchr(t + b, '\n', n - b);
            const size_t e = nl ? static_cast<size_t>(static_cast<const char*>(nl) - t) : n;
            size_t k = b;
            while (k < e && std::isspace(static_cast<unsigned char>(t[k]))) ++k;
            if (k < e && t[k] == '$') dollar_.push_back(lineBegin_.size());
            lineBegin_.push_back(b);
            lineEnd_.push_back(e);
            b = e + 1;
        }
    }

    const std::string& path() const { return path_; }

    /// $Name ... $EndName as rows; no rows when the file has no such
    /// section (an error if `required`)
    SectionRows section(const std::string& name, bool required) const
    {
        const std::string open = "$" + name, close = "$End" + name;
        for (size_t a = 0; a < dollar_.size(); ++a)
        {
            if (leadToken(dollar_[a]) != open) continue;
            for (size_t z = a + 1; z < dollar_.size(); ++z)
                if (leadToken(dollar_[z]) == close) return tokenise(dollar_[a] + 1, dollar_[z], open);
            raise(Msg::Unterminated, {open, path_});
        }
        if (required) raise(Msg::MissingSection, {path_, open});
        return SectionRows{};
    }

private:
    std::string_view leadToken(size_t line) const
    {
        const char* s = text_.data() + lineBegin_[line];
        const char* e = text_.data() + lineEnd_[line];
        while (s < e && std::isspace(static_cast<unsigned char>(*s))) ++s;
        const char* b = s;
        while (s < e && !std::isspace(static_cast<unsigned char>(*s))) ++s;
        return std::string_view(b, static_cast<size_t>(s - b));
    }

    /// lines [lo, hi) split into tokens on the host's threads: each part
    /// tokenises its own lines, then the parts are joined in order
    SectionRows tokenise(size_t lo, size_t hi, const std::string& open) const
    {
        SectionRows out;
        out.label = open + " in " + path_;
        const int64_t nLines = static_cast<int64_t>(hi - lo);
        const int64_t parts = std::max<int64_t>(1, std::min<int64_t>(64, nLines / 8192));
        struct Part
        {
            std::vector<std::string_view> tok;
            std::vector<size_t> end;
        };
        std::vector<Part> part(static_cast<size_t>(parts));
        parallelChunks(parts, 1, [&](int64_t pb, int64_t pe) {
            for (int64_t q = pb; q < pe; ++q)
            {
                Part& P = part[static_cast<size_t>(q)];
                const size_t l0 = lo + static_cast<size_t>(nLines * q / parts);
                const size_t l1 = lo + static_cast<size_t>(nLines * (q + 1) / parts);
                P.end.reserve(l1 - l0);
                for (size_t l = l0; l < l1; ++l)
                {
                    const char* s = text_.data() + lineBegin_[l];
                    const char* e = text_.data() + lineEnd_[l];
                    const size_t before = P.tok.size();
                    while (s < e)
                    {
                        while (s < e && isBlank(*s)) ++s;
                        const char* b = s;
                        while (s < e && !isBlank(*s)) ++s;
                        if (s > b) P.tok.emplace_back(b, static_cast<size_t>(s - b));
                    }
                    if (P.tok.size() > before) P.end.push_back(P.tok.size());
                }
            }
        });
        std::vector<size_t> tokAt(part.size() + 1, 0), rowAt(part.size() + 1, 0);
        for (size_t q = 0; q < part.size(); ++q)
        {
            tokAt[q + 1] = tokAt[q] + part[q].tok.size();
            rowAt[q + 1] = rowAt[q] + part[q].end.size();
        }
        out.tokens.resize(tokAt.back());
        out.rowEnd.resize(rowAt.back());
        parallelChunks(parts, 1, [&](int64_t pb, int64_t pe) {
            for (int64_t q = pb; q < pe; ++q)
            {
                const size_t u = static_cast<size_t>(q);
                std::copy(part[u].tok.begin(), part[u].tok.end(), out.tokens.begin() + static_cast<long>(tokAt[u]));
                for (size_t r = 0; r < part[u].end.size(); ++r) out.rowEnd[rowAt[u] + r] = tokAt[u] + part[u].end[r];
                std::vector<std::string_view>().swap(part[u].tok);
            }
        });
        return out;
    }

    std::string path_, text_;
    std::vector<size_t> lineBegin_, lineEnd_;
    std::vector<size_t> dollar_;  // lines that open with '$'
};

// ---------------------------------------------------------------------------
// element types (gmsh numbering)
// ---------------------------------------------------------------------------

enum : int
{
    kLine = 1, kTriangle = 2, kQuad = 3, kTet = 4, kHex = 5, kPrism = 6, kPyramid = 7
};

/// nodes of a first-order element of `type`; 0 for anything else
int nodeCount(int type)
{
    static constexpr int counts[] = {0, 2, 3, 4, 4, 8, 6, 5};
    return type >= kLine && type <= kPyramid ? counts[type] : 0;
}

bool isSurface(int type) { return type == kTriangle || type == kQuad; }
bool isVolume(int type) { return type == kTet || type == kHex || type == kPrism; }

// ---------------------------------------------------------------------------
// the readers
// ---------------------------------------------------------------------------

struct Format
{
    double version = 0;
    bool blocked = false;  // 4.x: nodes and elements come in entity blocks
};

Format readFormat(const MshText& f)
{
    const SectionRows s = f.section("MeshFormat", true);
    Cursor cur(s);
    const Row r = cur.next();
    if (r.n < 2) raise(Msg::BadFormatRow, {f.path()});
    Format fm;
    fm.version = parseReal(r[0], "$MeshFormat");
    if (parseInt(r[1], "$MeshFormat") != 0) raise(Msg::BinaryFile, {f.path()});
    const bool v22 = std::abs(fm.version - 2.2) < 1e-9;
    if (!v22 && !(fm.version >= 4.0)) raise(Msg::UnsupportedVersion, {std::string(r[0])});
    fm.blocked = fm.version >= 3.0;
    return fm;
}

/// names of the dimension-2 physical groups, by group tag
std::map<long, std::string> readSurfaceGroupNames(const MshText& f)
{
    std::map<long, std::string> names;
    const SectionRows s = f.section("PhysicalNames", false);
    if (!s.rows()) return names;
    Cursor cur(s);
    const long count = parseInt(cur.next()[0], "$PhysicalNames");
    for (long k = 0; k < count; ++k)
    {
        const Row r = cur.next();
        if (r.n < 3) raise(Msg::BadGroupRow);
        const long dim = parseInt(r[0], "$PhysicalNames");
        const long group = parseInt(r[1], "$PhysicalNames");
        // the name may hold blanks: its tokens are joined without them, and
        // the quotes dropped
        std::string name;
        for (size_t i = 2; i < r.n; ++i)
            for (char c : r[i])
                if (c != '"') name += c;
        if (name.empty()) raise(Msg::UnnamedGroup, {str(group)});
        if (dim == 2) names[group] = std::move(name);
    }
    return names;
}

/// Node tags and coordinates in file order; a tag of 0 marks a node written
/// without one.
struct NodeList
{
    std::vector<long> tag;
    std::vector<Vec> xyz;
};

Vec parseXyz(const Row& r, size_t col)
{
    return Vec{parseReal(r[col], "$Nodes"), parseReal(r[col + 1], "$Nodes"), parseReal(r[col + 2], "$Nodes")};
}

/// `count` coordinate rows from the cursor, decoded in parallel into `out`
/// from position `at`; with fewer rows left, those present are decoded (so
/// a bad one is reported first) and the missing one is the ran-out error.
template <class Decode>
void decodeRows(Cursor& cur, long count, Decode&& decode)
{
    const long have = std::max(0L, std::min(count, static_cast<long>(cur.left())));
    parallelChunks(have, 1 << 14, [&](int64_t lo, int64_t hi) {
        for (int64_t i = lo; i < hi; ++i) decode(i, cur.ahead(static_cast<size_t>(i)));
    });
    cur.skip(static_cast<size_t>(have));
    if (have < count) cur.next();
}

NodeList readNodeList(const MshText& f, const Format& fm)
{
    const SectionRows s = f.section("Nodes", true);
    if (!s.rows()) raise(Msg::EmptyNodes, {f.path()});
    Cursor cur(s);
    NodeList nl;
    long declared = 0;
    if (!fm.blocked)
    {
        // 2.2: a count, then "tag x y z" rows
        declared = parseInt(cur.next()[0], "$Nodes");
        const size_t want = static_cast<size_t>(std::max(0L, std::min(declared, static_cast<long>(cur.left()))));
        nl.tag.resize(want);
        nl.xyz.resize(want);
        decodeRows(cur, declared, [&](int64_t i, const Row& r) {
            if (r.n < 4) raise(Msg::BadNodeRow, {f.path()});
            nl.tag[static_cast<size_t>(i)] = parseInt(r[0], "$Nodes");
            nl.xyz[static_cast<size_t>(i)] = parseXyz(r, 1);
        });
    }
    else
    {
        // 4.x: "numBlocks numNodes firstTag ..." then blocks of
        // "dim entity parametric count [minTag maxTag]"; a block header
        // with the tag range puts the coordinates first and tag rows (when
        // the range is not a single tag) after them, one without puts one
        // tag row per node before the coordinates
        const Row h = cur.next();
        if (h.n < 4) raise(Msg::BadNodesHeader, {f.path()});
        const long blocks = parseInt(h[0], "$Nodes header");
        declared = parseInt(h[1], "$Nodes header");
        const long firstTag = parseInt(h[2], "$Nodes header");
        for (long b = 0; b < blocks; ++b)
        {
            const Row bh = cur.next();
            if (bh.n < 4) raise(Msg::BadNodeBlockHeader, {f.path()});
            const long count = parseInt(bh[3], "$Nodes block");
            if (count <= 0) continue;
            const bool ranged = bh.n >= 6;
            const long lowTag = ranged ? parseInt(bh[4], "$Nodes block") : firstTag;
            const long highTag = ranged ? parseInt(bh[5], "$Nodes block") : firstTag;
            const size_t base = nl.xyz.size();
            std::vector<long> tags;
            auto takeTags = [&]() {
                long t = 0;
                while (static_cast<long>(tags.size()) < count && cur.nextTag(t)) tags.push_back(t);
            };
            auto takeCoordinates = [&]() {
                const size_t want = static_cast<size_t>(std::min(count, static_cast<long>(cur.left())));
                nl.xyz.resize(base + want);
                decodeRows(cur, count, [&](int64_t i, const Row& r) {
                    if (r.n < 3) raise(Msg::BadCoordinates);
                    nl.xyz[base + static_cast<size_t>(i)] = parseXyz(r, 0);
                });
            };
            if (ranged)
            {
                takeCoordinates();
                if (lowTag != highTag) takeTags();
                if (tags.empty())
                {
                    tags.resize(static_cast<size_t>(count));
                    std::iota(tags.begin(), tags.end(), lowTag);
                }
                else if (static_cast<long>(tags.size()) != count)
                    raise(Msg::NodeTagCountMismatch, {f.path(), str(static_cast<long>(tags.size())), str(count)});
            }
            else
            {
                takeTags();
                if (static_cast<long>(tags.size()) != count) tags.assign(static_cast<size_t>(count), 0);
                takeCoordinates();
            }
            nl.tag.insert(nl.tag.end(), tags.begin(), tags.end());
        }
    }
    if (static_cast<long>(nl.xyz.size()) != declared)
        raise(Msg::NodeCountMismatch, {str(declared), str(static_cast<long>(nl.xyz.size())), f.path()});
    return nl;
}

/// Points in ascending tag order and the map from a tag to its point.
class NodeIndex
{
public:
    NodeIndex(NodeList nl, const std::string& path)
    {
        const size_t n = nl.tag.size();
        // nodes written without a tag (tag <= 0) take, in file order, the
        // smallest positive tags no tagged node uses: walk the sorted used
        // tags once, handing out the gaps
        std::vector<long> used;
        used.reserve(n);
        for (long t : nl.tag)
            if (t > 0) used.push_back(t);
        if (used.size() < n)
        {
            std::sort(used.begin(), used.end());
            used.erase(std::unique(used.begin(), used.end()), used.end());
            size_t u = 0;
            long candidate = 1;
            for (long& t : nl.tag)
            {
                if (t > 0) continue;
                while (u < used.size() && used[u] < candidate) ++u;
                while (u < used.size() && used[u] == candidate)
                {
                    ++candidate;
                    ++u;
                }
                t = candidate++;
            }
        }
        // points ordered by tag (file order kept among equal tags, which
        // are then refused)
        std::vector<size_t> order(n);
        std::iota(order.begin(), order.end(), size_t(0));
        const bool sorted = std::is_sorted(nl.tag.begin(), nl.tag.end());
        if (!sorted)
            std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return nl.tag[a] < nl.tag[b]; });
        points.resize(n);
        tags_.resize(n);
        dense_ = true;
        for (size_t i = 0; i < n; ++i)
        {
            const size_t k = order[i];
            tags_[i] = nl.tag[k];
            points[i] = nl.xyz[k];
            if (i > 0 && tags_[i] == tags_[i - 1]) raise(Msg::DuplicateNodeTag, {str(tags_[i]), path});
            dense_ = dense_ && tags_[i] == static_cast<long>(i) + 1;
        }
    }

    /// the point of node `tag`; false if no node has it
    bool find(long tag, int64_t& point) const
    {
        if (dense_)
        {
            if (tag < 1 || tag > static_cast<long>(tags_.size())) return false;
            point = tag - 1;
            return true;
        }
        const auto it = std::lower_bound(tags_.begin(), tags_.end(), tag);
        if (it == tags_.end() || *it != tag) return false;
        point = static_cast<int64_t>(it - tags_.begin());
        return true;
    }

    std::vector<Vec> points;

private:
    std::vector<long> tags_;  // ascending, one per point
    bool dense_ = true;       // the tags are 1..n
};

/// 4.x: the physical group of each surface entity, from $EntityNames and
/// then $Entities (which wins where both name one)
std::map<long, long> readSurfaceEntityGroups(const MshText& f)
{
    std::map<long, long> group;
    {
        const SectionRows s = f.section("EntityNames", false);
        if (s.rows())
        {
            Cursor cur(s);
            const long count = parseInt(cur.next()[0], "$EntityNames");
            for (long k = 0; k < count; ++k)
            {
                const Row r = cur.next();
                if (r.n < 4) raise(Msg::BadEntityNameRow);
                if (parseInt(r[0], "$EntityNames") == 2)
                    group[parseInt(r[1], "$EntityNames")] = parseInt(r[2], "$EntityNames");
            }
        }
    }
    const SectionRows s = f.section("Entities", false);
    if (!s.rows()) return group;
    Cursor cur(s);
    const Row h = cur.next();
    if (h.n < 4) raise(Msg::BadEntitiesHeader);
    long perDim[4];
    for (size_t d = 0; d < 4; ++d) perDim[d] = parseInt(h[d], "$Entities");
    // points, curves, surfaces, volumes; a surface row is
    // "tag minX minY minZ maxX maxY maxZ nGroups group..."
    for (int d = 0; d < 4; ++d)
        for (long k = 0; k < perDim[d]; ++k)
        {
            const Row r = cur.next();
            if (d != 2) continue;
            if (r.n < 8) raise(Msg::BadSurfaceEntity);
            const long entity = parseInt(r[0], "$Entities");
            if (parseInt(r[7], "$Entities") <= 0) continue;
            if (r.n < 9) raise(Msg::BadSurfaceEntity);
            group[entity] = parseInt(r[8], "$Entities");
        }
    return group;
}

/// Where an element row's data lie: its type, physical group, and the
/// column of its first node.
struct ElementRow
{
    Row row;
    int type;
    int col;
    long group;
};

/// The layout pass: every element row's shape checked, in file order.  The
/// rows point into `s`, which the caller keeps.
std::vector<ElementRow> layoutElements(const MshText& f, const SectionRows& s, const Format& fm,
                                       const std::map<long, long>& entityGroup)
{
    if (!s.rows()) raise(Msg::EmptyElements, {f.path()});
    Cursor cur(s);
    std::vector<ElementRow> out;
    if (!fm.blocked)
    {
        // 2.2: "number type nTags tag... node..." per row; the first tag is
        // the physical group
        const long declared = parseInt(cur.next()[0], "$Elements");
        const size_t have = static_cast<size_t>(std::max(0L, std::min(declared, static_cast<long>(cur.left()))));
        out.resize(have);
        parallelChunks(static_cast<int64_t>(have), 1 << 13, [&](int64_t lo, int64_t hi) {
            for (int64_t i = lo; i < hi; ++i)
            {
                const Row r = cur.ahead(static_cast<size_t>(i));
                if (r.n < 3) raise(Msg::BadElementRow, {f.path()});
                const int type = static_cast<int>(parseInt(r[1], "$Elements"));
                const int nodes = nodeCount(type);
                if (nodes == 0) raise(Msg::NotFirstOrder, {str(type), f.path()});
                const long nTags = parseInt(r[2], "$Elements");
                if (3 + nTags < 0) raise(Msg::BadElementRow, {f.path()});
                if (static_cast<long>(r.n) < 3 + nTags + nodes) raise(Msg::ShortElementRow, {f.path()});
                const long group = nTags > 0 ? parseInt(r[3], "$Elements") : 0;
                out[static_cast<size_t>(i)] = ElementRow{r, type, static_cast<int>(3 + nTags), group};
            }
        });
        cur.skip(have);
        if (static_cast<long>(have) < declared) cur.next();
        return out;
    }
    // 4.x: "numBlocks numElements ..." then blocks of
    // "dim entity type count", each followed by its rows; the first row's
    // width says whether the rows start with the element's own tag
    const Row h = cur.next();
    if (h.n < 4) raise(Msg::BadElementsHeader, {f.path()});
    const long blocks = parseInt(h[0], "$Elements header");
    const long declared = parseInt(h[1], "$Elements header");
    long seen = 0;
    for (long b = 0; b < blocks; ++b)
    {
        const Row bh = cur.next();
        if (bh.n < 4) raise(Msg::BadElementBlockHeader, {f.path()});
        const long entity = parseInt(bh[1], "$Elements block");
        const int type = static_cast<int>(parseInt(bh[2], "$Elements block"));
        const long count = parseInt(bh[3], "$Elements block");
        const int nodes = nodeCount(type);
        if (nodes == 0) raise(Msg::NotFirstOrder, {str(type), f.path()});
        const auto g = entityGroup.find(entity);
        const long group = g != entityGroup.end() ? g->second : 0;
        if (count <= 0) continue;
        const long have = std::min(count, static_cast<long>(cur.left()));
        int col = 0;
        if (have > 0)
        {
            const long width = static_cast<long>(cur.ahead(0).n);
            if (width == nodes + 1) col = 1;
            else if (width != nodes) raise(Msg::ElementWidth, {str(width), str(nodes), str(nodes + 1)});
        }
        const size_t base = out.size();
        out.resize(base + static_cast<size_t>(have));
        parallelChunks(have, 1 << 13, [&](int64_t lo, int64_t hi) {
            for (int64_t i = lo; i < hi; ++i)
            {
                const Row r = cur.ahead(static_cast<size_t>(i));
                if (static_cast<long>(r.n) != nodes + col) raise(Msg::ElementWidthChanged, {f.path()});
                out[base + static_cast<size_t>(i)] = ElementRow{r, type, col, group};
            }
        });
        cur.skip(static_cast<size_t>(have));
        seen += have;
        if (have < count) cur.next();
    }
    if (seen != declared) raise(Msg::ElementCountMismatch, {str(declared), str(seen), f.path()});
    return out;
}

/// The decode pass: one element's nodes as points.
struct DecodedElement
{
    int type;
    int n;
    long group;
    int64_t pt[8];
};

}  // namespace

Mesh readGmsh(const std::string& path, const std::map<std::string, std::string>& patchTypes)
{
    const MshText f(path);
    const Format fm = readFormat(f);
    const std::map<long, std::string> groupName = readSurfaceGroupNames(f);
    const NodeIndex nodes(readNodeList(f, fm), path);
    const std::map<long, long> entityGroup = fm.blocked ? readSurfaceEntityGroups(f) : std::map<long, long>{};
    const SectionRows elementRows = f.section("Elements", true);
    const std::vector<ElementRow> rows = layoutElements(f, elementRows, fm, entityGroup);

    std::vector<DecodedElement> dec(rows.size());
    parallelChunks(static_cast<int64_t>(rows.size()), 1 << 13, [&](int64_t lo, int64_t hi) {
        for (int64_t i = lo; i < hi; ++i)
        {
            const ElementRow& er = rows[static_cast<size_t>(i)];
            DecodedElement& d = dec[static_cast<size_t>(i)];
            d.type = er.type;
            d.n = nodeCount(er.type);
            d.group = er.group;
            for (int k = 0; k < d.n; ++k)
            {
                const long tag = parseInt(er.row[static_cast<size_t>(er.col + k)], "$Elements");
                if (!nodes.find(tag, d.pt[k])) raise(Msg::UnknownNode, {str(tag)});
            }
            // a node given twice in a row of the connectivity
            for (int k = 1; k < d.n; ++k)
                if (d.pt[k] == d.pt[k - 1]) raise(Msg::RepeatedNode, {str(d.type)});
            if (d.type == kPyramid) raise(Msg::Pyramid);
        }
    });

    // volumes become cells; grouped surface elements name the boundary
    // faces they cover (the first element of a face decides)
    std::vector<int32_t> types;
    std::vector<int64_t> offsets{0}, verts;
    types.reserve(dec.size());
    offsets.reserve(dec.size() + 1);
    verts.reserve(8 * dec.size());
    SurfaceNames surfaceNames;
    for (const DecodedElement& d : dec)
    {
        if (isVolume(d.type))
        {
            types.push_back(d.type);
            verts.insert(verts.end(), d.pt, d.pt + d.n);
            offsets.push_back(static_cast<int64_t>(verts.size()));
        }
        else if (isSurface(d.type))
        {
            const auto g = groupName.find(d.group);
            if (g == groupName.end()) continue;
            std::array<int64_t, 5> key;
            key.fill(-1);
            std::copy(d.pt, d.pt + d.n, key.begin());
            std::sort(key.begin(), key.begin() + d.n);
            surfaceNames.emplace(key, g->second);
        }
    }
    if (types.empty()) raise(Msg::NoVolumes, {path});
    return meshFromCells(nodes.points, types, offsets, verts, surfaceNames, patchTypes);
}

}  // namespace cfg
