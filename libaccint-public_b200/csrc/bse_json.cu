// Native loader of Basis Set Exchange JSON ("complete" or "minimal" schema) into
// a lai_basis: lai_basis_from_bse_json.  Host code only.
//
// Shell expansion follows the reference's BSE reader (src/shared/data/
// bse_json_parser.cpp:27-87): for every element shell, a single-l entry gives one
// contracted shell per coefficient column over ALL listed exponents, a multi-l
// (SP) entry gives one shell per angular momentum with its own column, and
// all-zero columns (general-contraction padding) are skipped.  Atoms are expanded
// in the order given, shells in file order; the raw coefficients are normalized by
// lai_basis_create exactly as for any other basis.  The schema check and the error
// cases (malformed text, no "elements", an element missing from the file) are the
// reference parser's (:90-140).
//
// The JSON reader below is a small recursive-descent parser of RFC 8259 text
// (objects, arrays, strings with escapes, numbers, true/false/null); BSE stores
// exponents and coefficients as strings, converted with strtod like the
// reference's std::stod.
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "engine_internal.h"

using namespace lai::host;

namespace {

struct JValue {
  enum Kind { NUL, BOOL, NUM, STR, ARR, OBJ } kind = NUL;
  bool b = false;
  double num = 0.0;
  std::string str;
  std::vector<JValue> arr;
  std::vector<std::pair<std::string, JValue>> obj;
  const JValue* get(const char* key) const {
    if (kind != OBJ) return nullptr;
    for (const auto& kv : obj)
      if (kv.first == key) return &kv.second;
    return nullptr;
  }
};

class JParser {
 public:
  JParser(const char* s, size_t n) : p_(s), end_(s + n) {}
  bool parse(JValue& v, std::string& err) {
    if (!value(v, 0)) {
      err = err_;
      return false;
    }
    ws();
    if (p_ != end_) {
      err = "trailing characters after the JSON value";
      return false;
    }
    return true;
  }

 private:
  const char* p_;
  const char* end_;
  std::string err_;

  bool fail(const char* m) {
    if (err_.empty()) err_ = m;
    return false;
  }
  void ws() {
    while (p_ < end_ && (*p_ == ' ' || *p_ == '\t' || *p_ == '\n' || *p_ == '\r')) ++p_;
  }
  bool lit(const char* w) {
    const size_t n = std::strlen(w);
    if ((size_t)(end_ - p_) < n || std::strncmp(p_, w, n) != 0) return fail("invalid literal");
    p_ += n;
    return true;
  }
  static void utf8(unsigned cp, std::string& out) {
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
  bool hex4(unsigned& cp) {
    if (end_ - p_ < 4) return fail("truncated \\u escape");
    cp = 0;
    for (int i = 0; i < 4; ++i) {
      const char c = *p_++;
      cp <<= 4;
      if (c >= '0' && c <= '9') cp |= (unsigned)(c - '0');
      else if (c >= 'a' && c <= 'f') cp |= (unsigned)(c - 'a' + 10);
      else if (c >= 'A' && c <= 'F') cp |= (unsigned)(c - 'A' + 10);
      else return fail("invalid \\u escape");
    }
    return true;
  }
  bool string(std::string& out) {
    if (p_ >= end_ || *p_ != '"') return fail("expected a string");
    ++p_;
    while (p_ < end_ && *p_ != '"') {
      const char c = *p_++;
      if ((unsigned char)c < 0x20) return fail("control character in a string");
      if (c != '\\') {
        out += c;
        continue;
      }
      if (p_ >= end_) return fail("truncated escape");
      const char e = *p_++;
      switch (e) {
        case '"': out += '"'; break;
        case '\\': out += '\\'; break;
        case '/': out += '/'; break;
        case 'b': out += '\b'; break;
        case 'f': out += '\f'; break;
        case 'n': out += '\n'; break;
        case 'r': out += '\r'; break;
        case 't': out += '\t'; break;
        case 'u': {
          unsigned cp;
          if (!hex4(cp)) return false;
          if (cp >= 0xD800 && cp < 0xDC00) {  // surrogate pair
            unsigned lo;
            if (end_ - p_ < 2 || p_[0] != '\\' || p_[1] != 'u') return fail("unpaired surrogate");
            p_ += 2;
            if (!hex4(lo) || lo < 0xDC00 || lo >= 0xE000) return fail("unpaired surrogate");
            cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
          }
          utf8(cp, out);
          break;
        }
        default: return fail("invalid escape");
      }
    }
    if (p_ >= end_) return fail("unterminated string");
    ++p_;
    return true;
  }
  bool number(double& v) {
    const char* s = p_;
    if (p_ < end_ && *p_ == '-') ++p_;
    if (p_ >= end_ || !(*p_ >= '0' && *p_ <= '9')) return fail("invalid number");
    while (p_ < end_ && ((*p_ >= '0' && *p_ <= '9') || *p_ == '.' || *p_ == 'e' || *p_ == 'E' ||
                         *p_ == '+' || *p_ == '-'))
      ++p_;
    const std::string tok(s, p_);
    char* q = nullptr;
    v = std::strtod(tok.c_str(), &q);
    if (!q || *q) return fail("invalid number");
    return true;
  }
  bool value(JValue& v, int depth) {
    if (depth > 64) return fail("nesting too deep");
    ws();
    if (p_ >= end_) return fail("unexpected end of text");
    const char c = *p_;
    if (c == '{') {
      ++p_;
      v.kind = JValue::OBJ;
      ws();
      if (p_ < end_ && *p_ == '}') {
        ++p_;
        return true;
      }
      for (;;) {
        ws();
        std::string k;
        if (!string(k)) return false;
        ws();
        if (p_ >= end_ || *p_ != ':') return fail("expected ':'");
        ++p_;
        v.obj.emplace_back(std::move(k), JValue());
        if (!value(v.obj.back().second, depth + 1)) return false;
        ws();
        if (p_ < end_ && *p_ == ',') {
          ++p_;
          continue;
        }
        if (p_ < end_ && *p_ == '}') {
          ++p_;
          return true;
        }
        return fail("expected ',' or '}'");
      }
    }
    if (c == '[') {
      ++p_;
      v.kind = JValue::ARR;
      ws();
      if (p_ < end_ && *p_ == ']') {
        ++p_;
        return true;
      }
      for (;;) {
        v.arr.emplace_back();
        if (!value(v.arr.back(), depth + 1)) return false;
        ws();
        if (p_ < end_ && *p_ == ',') {
          ++p_;
          continue;
        }
        if (p_ < end_ && *p_ == ']') {
          ++p_;
          return true;
        }
        return fail("expected ',' or ']'");
      }
    }
    if (c == '"') {
      v.kind = JValue::STR;
      return string(v.str);
    }
    if (c == 't') {
      v.kind = JValue::BOOL;
      v.b = true;
      return lit("true");
    }
    if (c == 'f') {
      v.kind = JValue::BOOL;
      return lit("false");
    }
    if (c == 'n') {
      v.kind = JValue::NUL;
      return lit("null");
    }
    v.kind = JValue::NUM;
    return number(v.num);
  }
};

// A BSE number: a string such as "1.172000E+04" (or, leniently, a JSON number).
bool bse_number(const JValue& v, double& out) {
  if (v.kind == JValue::NUM) {
    out = v.num;
    return true;
  }
  if (v.kind != JValue::STR) return false;
  const char* s = v.str.c_str();
  char* q = nullptr;
  out = std::strtod(s, &q);
  if (q == s) return false;
  while (*q == ' ') ++q;
  return *q == 0;
}

struct RawShell {
  int l;
  std::vector<double> exps, coefs;
};

int expand_element(const JValue& el, int Z, std::vector<RawShell>& out) {
  const JValue* shells = el.get("electron_shells");
  if (!shells) return LAI_OK;  // an element without electron shells gives none
  if (shells->kind != JValue::ARR) return fail(LAI_EINVAL, "BSE JSON: electron_shells is not an array");
  for (const JValue& sh : shells->arr) {
    const JValue* ex = sh.get("exponents");
    const JValue* am = sh.get("angular_momentum");
    const JValue* co = sh.get("coefficients");
    if (!ex || !am || !co || ex->kind != JValue::ARR || am->kind != JValue::ARR || co->kind != JValue::ARR)
      return fail(LAI_EINVAL, "BSE JSON: element " + std::to_string(Z) + ": malformed shell");
    std::vector<double> e(ex->arr.size());
    for (size_t i = 0; i < e.size(); ++i)
      if (!bse_number(ex->arr[i], e[i]))
        return fail(LAI_EINVAL, "BSE JSON: element " + std::to_string(Z) + ": bad exponent");
    std::vector<int> ls;
    for (const JValue& a : am->arr) {
      if (a.kind != JValue::NUM) return fail(LAI_EINVAL, "BSE JSON: bad angular momentum");
      ls.push_back((int)a.num);
    }
    if (ls.empty()) return fail(LAI_EINVAL, "BSE JSON: shell without angular momentum");
    const size_t ncol = ls.size() == 1 ? co->arr.size() : std::min(ls.size(), co->arr.size());
    for (size_t c = 0; c < ncol; ++c) {
      const JValue& col = co->arr[c];
      if (col.kind != JValue::ARR || col.arr.size() != e.size())
        return fail(LAI_EINVAL, "BSE JSON: element " + std::to_string(Z) +
                                    ": coefficient column length differs from the exponents");
      RawShell r;
      r.l = ls.size() == 1 ? ls[0] : ls[c];
      r.exps = e;
      r.coefs.resize(e.size());
      bool nonzero = false;
      for (size_t i = 0; i < e.size(); ++i) {
        if (!bse_number(col.arr[i], r.coefs[i])) return fail(LAI_EINVAL, "BSE JSON: bad coefficient");
        nonzero = nonzero || r.coefs[i] != 0.0;
      }
      if (nonzero) out.push_back(std::move(r));
    }
  }
  return LAI_OK;
}

}  // namespace

extern "C" {

int lai_basis_from_bse_json(const char* json_text, size_t length, int natom, const int* Z, const double* xyz,
                            lai_basis** out) {
  if (!out) return fail(LAI_EINVAL, "lai_basis_from_bse_json: out is NULL");
  *out = nullptr;
  if (!json_text || natom < 0 || (natom > 0 && (!Z || !xyz)))
    return fail(LAI_EINVAL, "lai_basis_from_bse_json: null argument");
  JValue root;
  std::string err;
  JParser parser(json_text, length);
  if (!parser.parse(root, err)) return fail(LAI_EINVAL, "Failed to parse BSE JSON: " + err);
  if (const JValue* schema = root.get("molssi_bse_schema")) {
    if (const JValue* st = schema->get("schema_type")) {
      if (st->kind != JValue::STR || (st->str != "complete" && st->str != "minimal"))
        return fail(LAI_EINVAL, "Unsupported BSE schema type: " + (st->kind == JValue::STR ? st->str : "?") +
                                    " (expected 'complete' or 'minimal')");
    }
  }
  const JValue* elements = root.get("elements");
  if (!elements || elements->kind != JValue::OBJ) return fail(LAI_EINVAL, "BSE JSON missing 'elements' key");
  std::map<int, std::vector<RawShell>> per_element;
  for (int a = 0; a < natom; ++a) {
    if (per_element.count(Z[a])) continue;
    const JValue* el = elements->get(std::to_string(Z[a]).c_str());
    if (!el) return fail(LAI_EINVAL, "Element Z=" + std::to_string(Z[a]) + " not found in BSE JSON");
    std::vector<RawShell> sh;
    if (int rc = expand_element(*el, Z[a], sh)) return rc;
    per_element.emplace(Z[a], std::move(sh));
  }
  std::vector<int> l, np, atom;
  std::vector<double> ctr, ex, co;
  for (int a = 0; a < natom; ++a)
    for (const RawShell& s : per_element[Z[a]]) {
      l.push_back(s.l);
      np.push_back((int)s.exps.size());
      atom.push_back(a);
      ctr.insert(ctr.end(), xyz + 3 * a, xyz + 3 * a + 3);
      ex.insert(ex.end(), s.exps.begin(), s.exps.end());
      co.insert(co.end(), s.coefs.begin(), s.coefs.end());
    }
  return lai_basis_create((int)l.size(), l.data(), np.data(), ctr.data(), ex.data(), co.data(), atom.data(), 0,
                          out);
}

}  // extern "C"
