// JSON value, parser and writer (see json.h).
#include "json.h"

#include <charconv>
#include <cstdint>
#include <cmath>
#include <cstdlib>
#include <cstring>

namespace ontc {

const Json* Json::find(const std::string& key) const
{
  if (type_ != Type::Object) return nullptr;
  auto it = obj_.find(key);
  return it == obj_.end() ? nullptr : &it->second;
}

// Exponent field of the scientific form: sign, then at least two digits.
static void append_exponent(std::string& out, int e)
{
  out.push_back(e < 0 ? '-' : '+');
  unsigned a = (unsigned)(e < 0 ? -e : e);
  if (a < 10) {
    out.push_back('0');
    out.push_back((char)('0' + a));
  } else {
    out += std::to_string(a);
  }
}

// ---- Grisu2 shortest-digit generation --------------------------------------------------
// F. Loitsch, "Printing Floating-Point Numbers Quickly and Accurately with Integers"
// (PLDI 2010), section 5, with the boundary-rounding step that nudges the last digit
// towards the exact value.  The parameters (target exponent window [-60, -32], cached
// powers of ten every 8 decades from 1e-300, round-half-up 64x64 products, one-ulp safety
// margin on each boundary) fix which of several round-trip digit strings is printed, and
// are the ones the ONTC writer's JSON library uses, so the bytes match it.
namespace {

struct Fp {
  uint64_t f;
  int e;
};

Fp fp_mul(Fp x, Fp y)
{
  const unsigned __int128 p = (unsigned __int128)x.f * y.f + ((unsigned __int128)1 << 63);
  return {(uint64_t)(p >> 64), x.e + y.e + 64};
}

Fp fp_normalize(Fp x)
{
  while ((x.f >> 63) == 0) {
    x.f <<= 1;
    x.e--;
  }
  return x;
}

struct Pow10 {
  uint64_t f;
  int e;
  int k;
};

// 64-bit significands of 10^k, k = -300 + 8 i (i = 0..78), rounded to nearest:
// 10^k ~= f * 2^e with 2^63 <= f < 2^64.
const Pow10 kPow10[79] = {
    {0xAB70FE17C79AC6CAull, -1060, -300},
    {0xFF77B1FCBEBCDC4Full, -1034, -292},
    {0xBE5691EF416BD60Cull, -1007, -284},
    {0x8DD01FAD907FFC3Cull, -980, -276},
    {0xD3515C2831559A83ull, -954, -268},
    {0x9D71AC8FADA6C9B5ull, -927, -260},
    {0xEA9C227723EE8BCBull, -901, -252},
    {0xAECC49914078536Dull, -874, -244},
    {0x823C12795DB6CE57ull, -847, -236},
    {0xC21094364DFB5637ull, -821, -228},
    {0x9096EA6F3848984Full, -794, -220},
    {0xD77485CB25823AC7ull, -768, -212},
    {0xA086CFCD97BF97F4ull, -741, -204},
    {0xEF340A98172AACE5ull, -715, -196},
    {0xB23867FB2A35B28Eull, -688, -188},
    {0x84C8D4DFD2C63F3Bull, -661, -180},
    {0xC5DD44271AD3CDBAull, -635, -172},
    {0x936B9FCEBB25C996ull, -608, -164},
    {0xDBAC6C247D62A584ull, -582, -156},
    {0xA3AB66580D5FDAF6ull, -555, -148},
    {0xF3E2F893DEC3F126ull, -529, -140},
    {0xB5B5ADA8AAFF80B8ull, -502, -132},
    {0x87625F056C7C4A8Bull, -475, -124},
    {0xC9BCFF6034C13053ull, -449, -116},
    {0x964E858C91BA2655ull, -422, -108},
    {0xDFF9772470297EBDull, -396, -100},
    {0xA6DFBD9FB8E5B88Full, -369, -92},
    {0xF8A95FCF88747D94ull, -343, -84},
    {0xB94470938FA89BCFull, -316, -76},
    {0x8A08F0F8BF0F156Bull, -289, -68},
    {0xCDB02555653131B6ull, -263, -60},
    {0x993FE2C6D07B7FACull, -236, -52},
    {0xE45C10C42A2B3B06ull, -210, -44},
    {0xAA242499697392D3ull, -183, -36},
    {0xFD87B5F28300CA0Eull, -157, -28},
    {0xBCE5086492111AEBull, -130, -20},
    {0x8CBCCC096F5088CCull, -103, -12},
    {0xD1B71758E219652Cull, -77, -4},
    {0x9C40000000000000ull, -50, 4},
    {0xE8D4A51000000000ull, -24, 12},
    {0xAD78EBC5AC620000ull, 3, 20},
    {0x813F3978F8940984ull, 30, 28},
    {0xC097CE7BC90715B3ull, 56, 36},
    {0x8F7E32CE7BEA5C70ull, 83, 44},
    {0xD5D238A4ABE98068ull, 109, 52},
    {0x9F4F2726179A2245ull, 136, 60},
    {0xED63A231D4C4FB27ull, 162, 68},
    {0xB0DE65388CC8ADA8ull, 189, 76},
    {0x83C7088E1AAB65DBull, 216, 84},
    {0xC45D1DF942711D9Aull, 242, 92},
    {0x924D692CA61BE758ull, 269, 100},
    {0xDA01EE641A708DEAull, 295, 108},
    {0xA26DA3999AEF774Aull, 322, 116},
    {0xF209787BB47D6B85ull, 348, 124},
    {0xB454E4A179DD1877ull, 375, 132},
    {0x865B86925B9BC5C2ull, 402, 140},
    {0xC83553C5C8965D3Dull, 428, 148},
    {0x952AB45CFA97A0B3ull, 455, 156},
    {0xDE469FBD99A05FE3ull, 481, 164},
    {0xA59BC234DB398C25ull, 508, 172},
    {0xF6C69A72A3989F5Cull, 534, 180},
    {0xB7DCBF5354E9BECEull, 561, 188},
    {0x88FCF317F22241E2ull, 588, 196},
    {0xCC20CE9BD35C78A5ull, 614, 204},
    {0x98165AF37B2153DFull, 641, 212},
    {0xE2A0B5DC971F303Aull, 667, 220},
    {0xA8D9D1535CE3B396ull, 694, 228},
    {0xFB9B7CD9A4A7443Cull, 720, 236},
    {0xBB764C4CA7A44410ull, 747, 244},
    {0x8BAB8EEFB6409C1Aull, 774, 252},
    {0xD01FEF10A657842Cull, 800, 260},
    {0x9B10A4E5E9913129ull, 827, 268},
    {0xE7109BFBA19C0C9Dull, 853, 276},
    {0xAC2820D9623BF429ull, 880, 284},
    {0x80444B5E7AA7CF85ull, 907, 292},
    {0xBF21E44003ACDD2Dull, 933, 300},
    {0x8E679C2F5E44FF8Full, 960, 308},
    {0xD433179D9C8CB841ull, 986, 316},
    {0x9E19DB92B4E31BA9ull, 1013, 324},
};

int largest_pow10(uint32_t n, uint32_t& p)
{
  static const uint32_t tens[10] = {1u, 10u, 100u, 1000u, 10000u, 100000u, 1000000u, 10000000u, 100000000u,
                                    1000000000u};
  for (int d = 9; d > 0; d--)
    if (n >= tens[d]) {
      p = tens[d];
      return d + 1;
    }
  p = 1;
  return 1;
}

void round_last(std::string& buf, uint64_t dist, uint64_t delta, uint64_t rest, uint64_t ten_k)
{
  while (rest < dist && delta - rest >= ten_k && (rest + ten_k < dist || dist - rest > rest + ten_k - dist)) {
    buf.back()--;
    rest += ten_k;
  }
}

// Digits of positive finite v and the decimal exponent: v ~= digits * 10^exp10.
void grisu2(double v, std::string& digits, int& exp10)
{
  uint64_t bits;
  memcpy(&bits, &v, 8);
  const uint64_t E = bits >> 52, F = bits & ((1ull << 52) - 1);
  const int kBias = 1023 + 52;
  Fp w = E == 0 ? Fp{F, 1 - kBias} : Fp{F + (1ull << 52), (int)E - kBias};
  const bool lower_closer = F == 0 && E > 1;
  Fp m_plus = fp_normalize(Fp{2 * w.f + 1, w.e - 1});
  Fp m_minus = lower_closer ? Fp{4 * w.f - 1, w.e - 2} : Fp{2 * w.f - 1, w.e - 1};
  m_minus = Fp{m_minus.f << (m_minus.e - m_plus.e), m_plus.e};
  w = fp_normalize(w);

  // cached power c = 10^-k with the product exponent inside [-60, -32]
  const int f = -60 - m_plus.e - 1;
  const int k = (f * 78913) / (1 << 18) + (f > 0 ? 1 : 0);
  const int index = (300 + k + 7) / 8;
  const Pow10 c = kPow10[index];
  const Fp cw = fp_mul(w, Fp{c.f, c.e});
  const Fp cminus = fp_mul(m_minus, Fp{c.f, c.e});
  const Fp cplus = fp_mul(m_plus, Fp{c.f, c.e});
  const Fp M_minus{cminus.f + 1, cminus.e};
  const Fp M_plus{cplus.f - 1, cplus.e};
  exp10 = -c.k;

  uint64_t delta = M_plus.f - M_minus.f;
  uint64_t dist = M_plus.f - cw.f;
  const int sh = -M_plus.e;
  const uint64_t one = 1ull << sh;
  uint32_t p1 = (uint32_t)(M_plus.f >> sh);
  uint64_t p2 = M_plus.f & (one - 1);
  uint32_t pow10;
  int n = largest_pow10(p1, pow10);
  digits.clear();
  while (n > 0) {
    const uint32_t d = p1 / pow10;
    p1 %= pow10;
    digits.push_back((char)('0' + d));
    n--;
    const uint64_t rest = ((uint64_t)p1 << sh) + p2;
    if (rest <= delta) {
      exp10 += n;
      round_last(digits, dist, delta, rest, (uint64_t)pow10 << sh);
      return;
    }
    pow10 /= 10;
  }
  int m = 0;
  for (;;) {
    p2 *= 10;
    const uint64_t d = p2 >> sh;
    p2 &= one - 1;
    digits.push_back((char)('0' + d));
    m++;
    delta *= 10;
    dist *= 10;
    if (p2 <= delta) break;
  }
  exp10 -= m;
  round_last(digits, dist, delta, p2, one);
}

}  // namespace

std::string format_double(double v)
{
  if (!std::isfinite(v)) return "null";
  std::string out;
  if (std::signbit(v)) {
    out.push_back('-');
    v = -v;
  }
  if (v == 0.0) {
    out += "0.0";
    return out;
  }
  std::string digits;
  int exp10 = 0;
  grisu2(v, digits, exp10);
  const int k = (int)digits.size();  // number of significant digits
  const int n = k + exp10;           // decimal point position relative to the digit string
  const int kMinExp = -4, kMaxExp = 15;
  if (k <= n && n <= kMaxExp) {
    // integral value: digits, zero padding, ".0"
    out += digits;
    out.append((size_t)(n - k), '0');
    out += ".0";
  } else if (0 < n && n <= kMaxExp) {
    out += digits.substr(0, (size_t)n);
    out.push_back('.');
    out += digits.substr((size_t)n);
  } else if (kMinExp < n && n <= 0) {
    out += "0.";
    out.append((size_t)(-n), '0');
    out += digits;
  } else {
    out.push_back(digits[0]);
    if (k > 1) {
      out.push_back('.');
      out += digits.substr(1);
    }
    out.push_back('e');
    append_exponent(out, n - 1);
  }
  return out;
}

static void dump_string(std::string& out, const std::string& s)
{
  out.push_back('"');
  for (unsigned char c : s) {
    switch (c) {
      case '"': out += "\\\""; break;
      case '\\': out += "\\\\"; break;
      case '\b': out += "\\b"; break;
      case '\f': out += "\\f"; break;
      case '\n': out += "\\n"; break;
      case '\r': out += "\\r"; break;
      case '\t': out += "\\t"; break;
      default:
        if (c < 0x20) {
          char tmp[8];
          snprintf(tmp, sizeof(tmp), "\\u%04x", c);
          out += tmp;
        } else {
          out.push_back((char)c);
        }
    }
  }
  out.push_back('"');
}

void Json::dump_to(std::string& out) const
{
  switch (type_) {
    case Type::Null: out += "null"; break;
    case Type::Bool: out += b_ ? "true" : "false"; break;
    case Type::Int: out += std::to_string(i_); break;
    case Type::Uint: out += std::to_string(u_); break;
    case Type::Float: out += format_double(d_); break;
    case Type::String: dump_string(out, s_); break;
    case Type::Array: {
      out.push_back('[');
      for (size_t i = 0; i < arr_.size(); i++) {
        if (i) out.push_back(',');
        arr_[i].dump_to(out);
      }
      out.push_back(']');
      break;
    }
    case Type::Object: {
      out.push_back('{');
      bool first = true;
      for (const auto& kv : obj_) {
        if (!first) out.push_back(',');
        first = false;
        dump_string(out, kv.first);
        out.push_back(':');
        kv.second.dump_to(out);
      }
      out.push_back('}');
      break;
    }
  }
}

std::string Json::dump() const
{
  std::string out;
  dump_to(out);
  return out;
}

struct JsonParser {
  const char* p;
  const char* end;
  int depth = 0;

  void ws()
  {
    while (p < end && (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r')) p++;
  }
  bool lit(const char* s)
  {
    size_t n = strlen(s);
    if ((size_t)(end - p) < n || memcmp(p, s, n) != 0) return false;
    p += n;
    return true;
  }
  static int hexval(char c)
  {
    if (c >= '0' && c <= '9') return c - '0';
    if (c >= 'a' && c <= 'f') return c - 'a' + 10;
    if (c >= 'A' && c <= 'F') return c - 'A' + 10;
    return -1;
  }
  bool hex4(unsigned& v)
  {
    if (end - p < 4) return false;
    v = 0;
    for (int i = 0; i < 4; i++) {
      int h = hexval(p[i]);
      if (h < 0) return false;
      v = v * 16 + (unsigned)h;
    }
    p += 4;
    return true;
  }
  static void utf8(std::string& s, unsigned cp)
  {
    if (cp < 0x80) {
      s.push_back((char)cp);
    } else if (cp < 0x800) {
      s.push_back((char)(0xC0 | (cp >> 6)));
      s.push_back((char)(0x80 | (cp & 0x3F)));
    } else if (cp < 0x10000) {
      s.push_back((char)(0xE0 | (cp >> 12)));
      s.push_back((char)(0x80 | ((cp >> 6) & 0x3F)));
      s.push_back((char)(0x80 | (cp & 0x3F)));
    } else {
      s.push_back((char)(0xF0 | (cp >> 18)));
      s.push_back((char)(0x80 | ((cp >> 12) & 0x3F)));
      s.push_back((char)(0x80 | ((cp >> 6) & 0x3F)));
      s.push_back((char)(0x80 | (cp & 0x3F)));
    }
  }
  bool string(std::string& s)
  {
    if (p >= end || *p != '"') return false;
    p++;
    while (p < end) {
      unsigned char c = (unsigned char)*p++;
      if (c == '"') return true;
      if (c < 0x20) return false;
      if (c != '\\') {
        s.push_back((char)c);
        continue;
      }
      if (p >= end) return false;
      char e = *p++;
      switch (e) {
        case '"': s.push_back('"'); break;
        case '\\': s.push_back('\\'); break;
        case '/': s.push_back('/'); break;
        case 'b': s.push_back('\b'); break;
        case 'f': s.push_back('\f'); break;
        case 'n': s.push_back('\n'); break;
        case 'r': s.push_back('\r'); break;
        case 't': s.push_back('\t'); break;
        case 'u': {
          unsigned cp;
          if (!hex4(cp)) return false;
          if (cp >= 0xD800 && cp < 0xDC00) {
            unsigned lo;
            if (!lit("\\u") || !hex4(lo) || lo < 0xDC00 || lo >= 0xE000) return false;
            cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
          } else if (cp >= 0xDC00 && cp < 0xE000) {
            return false;
          }
          utf8(s, cp);
          break;
        }
        default: return false;
      }
    }
    return false;
  }
  bool number(Json& out)
  {
    const char* s = p;
    bool neg = false, frac = false;
    if (p < end && *p == '-') {
      neg = true;
      p++;
    }
    if (p >= end) return false;
    if (*p == '0') {
      p++;
    } else if (*p >= '1' && *p <= '9') {
      while (p < end && *p >= '0' && *p <= '9') p++;
    } else {
      return false;
    }
    if (p < end && *p == '.') {
      frac = true;
      p++;
      if (p >= end || !(*p >= '0' && *p <= '9')) return false;
      while (p < end && *p >= '0' && *p <= '9') p++;
    }
    if (p < end && (*p == 'e' || *p == 'E')) {
      frac = true;
      p++;
      if (p < end && (*p == '+' || *p == '-')) p++;
      if (p >= end || !(*p >= '0' && *p <= '9')) return false;
      while (p < end && *p >= '0' && *p <= '9') p++;
    }
    std::string tok(s, p);
    if (!frac) {
      if (neg) {
        int64_t v;
        auto r = std::from_chars(tok.data(), tok.data() + tok.size(), v);
        if (r.ec == std::errc()) {
          out = Json::make_int(v);
          return true;
        }
      } else {
        uint64_t v;
        auto r = std::from_chars(tok.data(), tok.data() + tok.size(), v);
        if (r.ec == std::errc()) {
          out = Json::make_uint(v);
          return true;
        }
      }
    }
    out = Json::make_float(strtod(tok.c_str(), nullptr));
    return true;
  }
  bool value(Json& out)
  {
    if (++depth > 512) return false;
    ws();
    if (p >= end) return false;
    bool ok = false;
    char c = *p;
    if (c == '{') {
      p++;
      out = Json::make_object();
      ws();
      if (p < end && *p == '}') {
        p++;
        ok = true;
      } else {
        while (true) {
          ws();
          std::string key;
          if (!string(key)) break;
          ws();
          if (p >= end || *p != ':') break;
          p++;
          Json v;
          if (!value(v)) break;
          out.obj_[key] = std::move(v);  // a repeated key keeps the last value
          ws();
          if (p < end && *p == ',') {
            p++;
            continue;
          }
          if (p < end && *p == '}') {
            p++;
            ok = true;
          }
          break;
        }
      }
    } else if (c == '[') {
      p++;
      out = Json::make_array();
      ws();
      if (p < end && *p == ']') {
        p++;
        ok = true;
      } else {
        while (true) {
          Json v;
          if (!value(v)) break;
          out.arr_.push_back(std::move(v));
          ws();
          if (p < end && *p == ',') {
            p++;
            continue;
          }
          if (p < end && *p == ']') {
            p++;
            ok = true;
          }
          break;
        }
      }
    } else if (c == '"') {
      std::string s;
      ok = string(s);
      if (ok) out = Json::make_string(std::move(s));
    } else if (c == 't') {
      ok = lit("true");
      if (ok) out = Json::make_bool(true);
    } else if (c == 'f') {
      ok = lit("false");
      if (ok) out = Json::make_bool(false);
    } else if (c == 'n') {
      ok = lit("null");
      if (ok) out = Json();
    } else {
      ok = number(out);
    }
    depth--;
    return ok;
  }
};

bool Json::parse(const char* begin, const char* end, Json& out)
{
  JsonParser ps{begin, end};
  if (!ps.value(out)) return false;
  ps.ws();
  return ps.p == end;
}

}  // namespace ontc
