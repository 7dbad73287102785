// Property files: the Eclipse-style INC text format and the GSLIB format
// (read_inc_file.cpp:8-193, property_writer.cpp:10-216).
//
// The reference reads with fscanf/sscanf on one thread. Here the file is read
// whole and its data part cut into chunks at line ends (a token, and a
// comment's rest of line, never crosses a line end); threads tokenise and
// convert their chunks, then the first `size` values are taken in file order.
// Conversions are the C library's: a token that strtof (strtol) consumes
// whole is converted by it, any other token by sscanf("%f") ("%d") exactly as
// the reference converts it. Writing formats chunks in parallel with the
// reference's printf conversions and writes them in order.
#include "engine_api.h"

#include <algorithm>
#include <cctype>
#include <clocale>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace hb
{
namespace
{
// The C library's numeric conversions run in the "C" locale (locale_keeper in
// the reference); this thread-local switch leaves other threads alone.
struct CLocale
{
    locale_t c = nullptr, old = nullptr;
    CLocale()
    {
        c = newlocale(LC_NUMERIC_MASK, "C", (locale_t)0);
        if (c) old = uselocale(c);
    }
    ~CLocale()
    {
        if (c)
        {
            uselocale(old);
            freelocale(c);
        }
    }
};

bool is_space(char ch) { return ch == ' ' || ch == '\t' || ch == '\n' || ch == '\r' || ch == '\v' || ch == '\f'; }

std::vector<char> read_all(const char *path, const char *who)
{
    FILE *f = fopen(path, "rb");
    if (!f) throw std::runtime_error(std::string(who) + ": Error opening file:" + path + ".");
    std::vector<char> buf;
    if (fseek(f, 0, SEEK_END) == 0)
    {
        const long sz = ftell(f);
        if (sz > 0) buf.reserve((size_t)sz + 1);
        rewind(f);
    }
    char tmp[1 << 16];
    size_t n;
    while ((n = fread(tmp, 1, sizeof(tmp), f)) > 0) buf.insert(buf.end(), tmp, tmp + n);
    const bool err = ferror(f) != 0;
    fclose(f);
    if (err) throw std::runtime_error(std::string(who) + ": Error reading file.");
    buf.push_back('\0');
    return buf;
}

// read_prop_name (read_inc_file.cpp:8-48): lines are read up to their end and
// the whitespace after them is skipped (fscanf "%1023[^\n]\n"); the first line
// whose first character is a letter is the property name. Returns the offset
// of the data. (An empty first line, on which the reference loops forever, is
// skipped like a blank one.)
size_t skip_header(const std::vector<char> &b, const char *who)
{
    const size_t end = b.size() - 1;
    size_t pos = 0;
    for (;;)
    {
        if (pos >= end) throw std::runtime_error(std::string(who) + ": Property name not found.");
        size_t e = pos;
        while (e < end && b[e] != '\n') ++e;
        const bool named = e > pos && isalpha(static_cast<unsigned char>(b[pos]));
        pos = e;
        while (pos < end && is_space(b[pos])) ++pos;
        if (named) return pos;
    }
}

enum TokKind
{
    TOK_VALUE,
    TOK_END,  // a token starting with '/'
    TOK_ERROR // a token the conversion rejects
};

template <typename T>
struct Chunk
{
    std::vector<T> vals;
    long long bad_at = -1; // index (in this chunk's values) of the first '/' or bad token
    TokKind bad_kind = TOK_VALUE;
    std::string bad_token;
};

// Tokens as fscanf("%255s") cuts them: whitespace-separated, at most 255
// characters (a longer run continues as the next token); a token starting
// with "--" skips the rest of its line.
template <typename T, typename Conv>
void parse_chunk(const char *p, const char *e, Chunk<T> &out, Conv conv)
{
    char tok[256];
    while (p < e)
    {
        while (p < e && is_space(*p)) ++p;
        if (p >= e) break;
        const char *s = p;
        while (p < e && !is_space(*p) && p - s < 255) ++p;
        const size_t len = (size_t)(p - s);
        if (len >= 2 && s[0] == '-' && s[1] == '-')
        {
            while (p < e && *p != '\n') ++p;
            continue;
        }
        std::memcpy(tok, s, len);
        tok[len] = '\0';
        if (s[0] == '/')
        {
            if (out.bad_at < 0)
            {
                out.bad_at = (long long)out.vals.size();
                out.bad_kind = TOK_END;
            }
            out.vals.push_back(T());
            continue;
        }
        T v;
        if (!conv(tok, len, v))
        {
            if (out.bad_at < 0)
            {
                out.bad_at = (long long)out.vals.size();
                out.bad_kind = TOK_ERROR;
                out.bad_token = tok;
            }
            v = T();
        }
        out.vals.push_back(v);
    }
}

bool conv_float(const char *tok, size_t len, float &v)
{
    char *end = nullptr;
    v = strtof(tok, &end);
    if (end == tok + len && len > 0) return true;
    return sscanf(tok, "%f", &v) == 1;
}

bool conv_int(const char *tok, size_t len, int &v)
{
    char *end = nullptr;
    const long x = strtol(tok, &end, 10);
    if (end == tok + len && len > 0 && x >= -2147483647L - 1 && x <= 2147483647L)
    {
        v = (int)x;
        return true;
    }
    return sscanf(tok, "%d", &v) == 1;
}

int io_threads() { return std::max(1, std::min(get_threads() > 0 ? get_threads() : 8, 64)); }

// The first `size` values of the data part, in file order.
template <typename T, typename Conv>
void parse_values(const std::vector<char> &b, size_t start, long long size, T *out, const char *who, Conv conv)
{
    const size_t end = b.size() - 1;
    const int nt = (int)std::min<long long>(io_threads(), std::max<long long>(1, (long long)(end - start) >> 16));
    std::vector<size_t> cut(nt + 1, end);
    cut[0] = start;
    for (int t = 1; t < nt; ++t)
    {
        size_t c = start + (end - start) * t / nt;
        while (c < end && b[c] != '\n') ++c;
        cut[t] = std::max(c, cut[t - 1]);
    }
    std::vector<Chunk<T>> ch(nt);
    {
        std::vector<std::thread> th;
        for (int t = 0; t < nt; ++t)
            th.emplace_back([&, t]() {
                CLocale loc;
                parse_chunk(b.data() + cut[t], b.data() + cut[t + 1], ch[t], conv);
            });
        for (auto &x : th) x.join();
    }
    long long have = 0;
    for (int t = 0; t < nt && have < size; ++t)
    {
        const Chunk<T> &c = ch[t];
        const long long take = std::min<long long>((long long)c.vals.size(), size - have);
        if (c.bad_at >= 0 && c.bad_at < take)
        {
            if (c.bad_kind == TOK_END) throw std::runtime_error(std::string(who) + ": Unexpected end of data.");
            throw std::runtime_error(std::string(who) + ": Error parsing '" + c.bad_token + "' string.");
        }
        std::copy(c.vals.begin(), c.vals.begin() + take, out + have);
        have += take;
    }
    if (have < size) throw std::runtime_error(std::string(who) + ": Unexpected end of file.");
}
} // namespace

void read_inc_float(const char *path, float undefined_value, long long size, float *data, unsigned char *mask)
{
    std::vector<char> b = read_all(path, "read_inc_file_float");
    const size_t start = skip_header(b, "read_prop_name");
    parse_values(b, start, size, data, "load_floats_into_vector", conv_float);
    if (mask)
        for (long long i = 0; i < size; ++i) mask[i] = data[i] == undefined_value ? 0 : 1;
}

void read_inc_byte(const char *path, int undefined_value, long long size, unsigned char *data, unsigned char *mask)
{
    std::vector<char> b = read_all(path, "read_inc_file_byte");
    const size_t start = skip_header(b, "read_prop_name");
    std::vector<int> v((size_t)size);
    parse_values(b, start, size, v.data(), "read_bytes", conv_int);
    for (long long i = 0; i < size; ++i)
    {
        data[i] = (unsigned char)v[i];
        mask[i] = v[i] == undefined_value ? 0 : 1;
    }
}

namespace
{
// Formats values [0, n) in parallel chunks with `fmt(i, buf)` (the bytes of
// value i) and writes them in order after `head`, then `tail`.
template <typename Fmt>
void write_formatted(const char *path, const std::string &head, long long n, const std::string &tail, Fmt fmt)
{
    FILE *f = fopen(path, "w+");
    if (!f) throw std::runtime_error(std::string("open_file_checked: Can't open file '") + path + "'.");
    const int nt = (int)std::min<long long>(io_threads(), std::max<long long>(1, n >> 14));
    std::vector<std::string> parts(nt);
    {
        std::vector<std::thread> th;
        for (int t = 0; t < nt; ++t)
            th.emplace_back([&, t]() {
                CLocale loc;
                const long long a = n * t / nt, z = n * (t + 1) / nt;
                std::string &s = parts[t];
                s.reserve((size_t)(z - a) * 14);
                char buf[64];
                for (long long i = a; i < z; ++i) s.append(buf, (size_t)fmt(i, buf));
            });
        for (auto &x : th) x.join();
    }
    bool ok = fwrite(head.data(), 1, head.size(), f) == head.size();
    for (auto &s : parts) ok = ok && fwrite(s.data(), 1, s.size(), f) == s.size();
    ok = ok && fwrite(tail.data(), 1, tail.size(), f) == tail.size();
    ok = (fclose(f) == 0) && ok;
    if (!ok) throw std::runtime_error(std::string("write: error writing '") + path + "'.");
}

// write_value (property_writer.cpp:19-27)
int fmt_double(double v, char *buf) { return snprintf(buf, 64, "%E\n", v); }
int fmt_byte(unsigned char v, char *buf) { return snprintf(buf, 64, "%d\n", (int)(char)v); }
} // namespace

void write_inc_float(const char *path, const char *name, const float *data, const unsigned char *mask,
                     long long size, float undefined_value, bool gslib)
{
    const std::string head = gslib ? std::string("HPGL saved GSLIB file\n1\n") + name + "\n" : std::string(name) + "\n";
    write_formatted(path, head, size, gslib ? "" : "/\n", [&](long long i, char *buf) {
        return fmt_double(mask[i] ? (double)data[i] : (double)undefined_value, buf);
    });
}

void write_inc_byte(const char *path, const char *name, const unsigned char *data, const unsigned char *mask,
                    long long size, unsigned char undefined_value, const std::vector<unsigned char> &remap,
                    bool gslib)
{
    const std::string head = gslib ? std::string("HPGL saved GSLIB file\n1\n") + name + "\n" : std::string(name) + "\n";
    // a category index beyond the remap table is written as it is
    write_formatted(path, head, size, gslib ? "" : "/\n", [&](long long i, char *buf) {
        return fmt_byte(mask[i] ? (data[i] < remap.size() ? remap[data[i]] : data[i]) : undefined_value, buf);
    });
}
} // namespace hb
