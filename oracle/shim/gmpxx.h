/* Minimal stand-in for GMP's C++ class mpz_class, written for this harness
 * (the GMP development headers are not installed on this machine).  It
 * stores a signed 128-bit integer, which is exact for every quantity the
 * exact-linear-algebra path touches: moduli below 2^32 and their products.
 * It is NOT GMP and offers none of its arbitrary-precision behaviour.
 * Test infrastructure only (oracle/_ref). */
#ifndef ORACLE_SHIM_GMPXX_H
#define ORACLE_SHIM_GMPXX_H
#include <iostream>
#include <string>
#include <cstdlib>

class mpz_class {
public:
	typedef __int128 rep;
	rep v;
	mpz_class () : v (0) {}
	mpz_class (int x) : v (x) {}
	mpz_class (unsigned int x) : v (x) {}
	mpz_class (long x) : v (x) {}
	mpz_class (unsigned long x) : v (x) {}
	mpz_class (long long x) : v (x) {}
	mpz_class (unsigned long long x) : v (x) {}
	mpz_class (double x) : v ((rep) x) {}
	mpz_class (float x) : v ((rep) x) {}
	mpz_class (const char *s) : v (0) { parse (s); }
	mpz_class (const std::string &s) : v (0) { parse (s.c_str ()); }
	void parse (const char *s) {
		bool neg = false; v = 0;
		while (*s == ' ') ++s;
		if (*s == '-') { neg = true; ++s; } else if (*s == '+') ++s;
		for (; *s >= '0' && *s <= '9'; ++s) v = v * 10 + (*s - '0');
		if (neg) v = -v;
	}
	unsigned long get_ui () const { return (unsigned long) (v < 0 ? -v : v); }
	long get_si () const { return (long) v; }
	double get_d () const { return (double) v; }
	std::string get_str (int base = 10) const {
		if (v == 0) return "0";
		rep t = v < 0 ? -v : v; std::string s;
		while (t > 0) { s.insert (s.begin (), (char) ('0' + (int) (t % base))); t /= base; }
		if (v < 0) s.insert (s.begin (), '-');
		return s;
	}
	mpz_class &operator += (const mpz_class &o) { v += o.v; return *this; }
	mpz_class &operator -= (const mpz_class &o) { v -= o.v; return *this; }
	mpz_class &operator *= (const mpz_class &o) { v *= o.v; return *this; }
	mpz_class &operator /= (const mpz_class &o) { v /= o.v; return *this; }
	mpz_class &operator %= (const mpz_class &o) { v %= o.v; return *this; }
	mpz_class &operator ++ () { ++v; return *this; }
	mpz_class &operator -- () { --v; return *this; }
	mpz_class operator - () const { mpz_class r; r.v = -v; return r; }
};

inline mpz_class mk_mpz (__int128 x) { mpz_class r; r.v = x; return r; }

/* The mixed-type operators below are restricted to built-in arithmetic
 * types, so that they never compete with the built-in operators for class
 * types that merely convert to an integer. */
template <class T> struct mpz_num { };
#define MPZ_NUM(T) template <> struct mpz_num<T> { typedef mpz_class mpz; typedef bool boolean; };
MPZ_NUM(char) MPZ_NUM(signed char) MPZ_NUM(unsigned char) MPZ_NUM(short) MPZ_NUM(unsigned short)
MPZ_NUM(int) MPZ_NUM(unsigned int) MPZ_NUM(long) MPZ_NUM(unsigned long)
MPZ_NUM(long long) MPZ_NUM(unsigned long long) MPZ_NUM(double) MPZ_NUM(float)
#undef MPZ_NUM

#define MPZ_BINOP(op) \
	inline mpz_class operator op (const mpz_class &a, const mpz_class &b) { return mk_mpz (a.v op b.v); } \
	template <class T> inline typename mpz_num<T>::mpz operator op (const mpz_class &a, T b) { return mk_mpz (a.v op mpz_class (b).v); } \
	template <class T> inline typename mpz_num<T>::mpz operator op (T a, const mpz_class &b) { return mk_mpz (mpz_class (a).v op b.v); }
MPZ_BINOP(+) MPZ_BINOP(-) MPZ_BINOP(*) MPZ_BINOP(/) MPZ_BINOP(%)
#undef MPZ_BINOP
#define MPZ_CMP(op) \
	inline bool operator op (const mpz_class &a, const mpz_class &b) { return a.v op b.v; } \
	template <class T> inline typename mpz_num<T>::boolean operator op (const mpz_class &a, T b) { return a.v op mpz_class (b).v; } \
	template <class T> inline typename mpz_num<T>::boolean operator op (T a, const mpz_class &b) { return mpz_class (a).v op b.v; }
MPZ_CMP(<) MPZ_CMP(>) MPZ_CMP(<=) MPZ_CMP(>=) MPZ_CMP(==) MPZ_CMP(!=)
#undef MPZ_CMP

inline std::ostream &operator << (std::ostream &o, const mpz_class &a) { return o << a.get_str (); }
// Formatted input as GMP's: white space skipped, an optional sign, decimal
// digits up to the first other character (left in the stream); failbit
// when no digit follows.
inline std::istream &operator >> (std::istream &i, mpz_class &a)
{
	std::istream::sentry se (i);
	if (!se) return i;
	std::string s;
	int c = i.peek ();
	if (c == '-' || c == '+') { s += (char) i.get (); c = i.peek (); }
	bool any = false;
	while (c >= '0' && c <= '9') { s += (char) i.get (); c = i.peek (); any = true; }
	if (!any) { i.setstate (std::ios::failbit); return i; }
	a.parse (s.c_str ());
	return i;
}
inline mpz_class abs (const mpz_class &a) { return a.v < 0 ? -a : a; }
#endif
