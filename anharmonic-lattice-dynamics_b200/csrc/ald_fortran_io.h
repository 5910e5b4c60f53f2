// gfortran's output edits, as the reference's output files are written
// with them (the rules are stated at the top of ald_writers.cpp).
#pragma once
#include <string>

namespace ald {
namespace fio {

std::string edit_I(int w, long long v);
std::string edit_F(int w, int d, double x);
std::string edit_E(int w, int d, double x);
std::string edit_G(int w, int d, double x);
std::string list_real(double x);  // one list-directed REAL(8) field, 25 characters
std::string list_int(long long v);  // one list-directed INTEGER field, 11 characters

// A list-directed record: items separated as write(u,*) separates them.
class ListRecord {
 public:
  ListRecord& i(long long v) { return item(list_int(v), false); }
  ListRecord& r(double v) { return item(list_real(v), false); }
  ListRecord& c(const char* t) { return item(t, true); }
  const std::string& str() const { return s_; }

 private:
  ListRecord& item(const std::string& t, bool chr) {
    if (!(chr && last_chr_) || s_.empty()) s_ += ' ';
    s_ += t;
    last_chr_ = chr;
    return *this;
  }
  std::string s_;
  bool last_chr_ = false;
};

}  // namespace fio
}  // namespace ald
