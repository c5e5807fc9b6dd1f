// Replay stand-in for LAMMPS (declarations and semantics in lammps/lammps.h).
// Test infrastructure only: lets the reference's ms-stem-fem-md driver run
// with its "MD" replaced by a cyclic replay of LAMMPS data files.
#include "lammps/atom.h"
#include "lammps/comm.h"
#include "lammps/error.h"
#include "lammps/input.h"
#include "lammps/lammps.h"
#include "lammps/library.h"
#include "lammps/memory.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

namespace LAMMPS_NS {

struct Replay {
  std::vector<std::string> files;  // MSF_MD_REPLAY list
  size_t next = 0;                 // index of the file the next run loads
  std::vector<tagint> tag;
  std::vector<int> type;
  std::vector<double> xyz;
  std::vector<double*> rows;
};

namespace {

bool starts_with(const std::string& s, const char* p) { return s.compare(0, std::strlen(p), p) == 0; }

// LAMMPS data file, atom style atomic: header with "N atoms" and the
// "lo hi xlo xhi" box lines, then an "Atoms" section of "id type x y z"
// lines (image flags, if present, ignored).  Atoms are stored by id.
bool read_data(LAMMPS* lmp, const std::string& path) {
  std::ifstream in(path.c_str());
  if (!in) {
    std::fprintf(stderr, "lammps replay: cannot open %s\n", path.c_str());
    return false;
  }
  Replay& r = *lmp->replay;
  std::string line;
  long long n = -1;
  bool atoms = false;
  long long seen = 0;
  while (std::getline(in, line)) {
    const size_t hash = line.find('#');
    std::string body = hash == std::string::npos ? line : line.substr(0, hash);
    std::istringstream ls(body);
    if (!atoms) {
      std::vector<std::string> tok;
      std::string t;
      while (ls >> t) tok.push_back(t);
      if (tok.empty()) continue;
      if (tok.size() >= 2 && tok[1] == "atoms") n = std::atoll(tok[0].c_str());
      for (int d = 0; d < 3; ++d) {
        static const char* lo[3] = {"xlo", "ylo", "zlo"};
        if (tok.size() >= 4 && tok[2] == lo[d]) {
          lmp->boxlo[d] = std::atof(tok[0].c_str());
          lmp->boxhi[d] = std::atof(tok[1].c_str());
        }
      }
      if (tok[0] == "Atoms") {
        if (n < 0) return false;
        r.tag.assign(n, 0);
        r.type.assign(n, 0);
        r.xyz.assign(3 * n, 0.0);
        atoms = true;
      }
      continue;
    }
    long long id;
    int ty;
    double x, y, z;
    if (!(ls >> id >> ty >> x >> y >> z)) continue;
    if (id < 1 || id > n) return false;
    r.tag[id - 1] = (tagint)id;
    r.type[id - 1] = ty;
    r.xyz[3 * (id - 1) + 0] = x;
    r.xyz[3 * (id - 1) + 1] = y;
    r.xyz[3 * (id - 1) + 2] = z;
    ++seen;
    if (seen == n) break;
  }
  if (seen != n) {
    std::fprintf(stderr, "lammps replay: %s holds %lld of %lld atoms\n", path.c_str(), seen, n);
    return false;
  }
  r.rows.resize(n);
  for (long long i = 0; i < n; ++i) r.rows[i] = &r.xyz[3 * i];
  Atom* a = lmp->atom;
  a->natoms = n;
  a->nlocal = (int)n;
  a->tag = r.tag.data();
  a->type = r.type.data();
  a->x = r.rows.data();
  return true;
}

char* run_command(LAMMPS* lmp, const char* command) {
  std::istringstream ls(command ? command : "");
  std::string word;
  if (!(ls >> word)) return 0;
  if (word == "read_data") {
    std::string path;
    ls >> path;
    if (!read_data(lmp, path)) std::exit(2);
  } else if (word == "run") {
    Replay& r = *lmp->replay;
    if (r.files.empty()) {
      std::fprintf(stderr, "lammps replay: run without MSF_MD_REPLAY\n");
      std::exit(2);
    }
    if (!read_data(lmp, r.files[r.next])) std::exit(2);
    r.next = (r.next + 1) % r.files.size();
  }
  return 0;
}

}  // namespace

LAMMPS::LAMMPS(int, char**, MPI_Comm communicator)
    : input(0), atom(new Atom), comm(new Comm), error(new Error), memory(new Memory),
      world(communicator), replay(new Replay), triclinic(0) {
  input = new Input(this);
  for (int d = 0; d < 3; ++d) boxlo[d] = boxhi[d] = 0.0;
  if (const char* list = std::getenv("MSF_MD_REPLAY")) {
    std::ifstream in(list);
    std::string line;
    while (std::getline(in, line)) {
      std::istringstream ls(line);
      std::string p;
      if (ls >> p) replay->files.push_back(p);
    }
  }
}

LAMMPS::~LAMMPS() {
  delete input;
  delete atom;
  delete comm;
  delete error;
  delete memory;
  delete replay;
}

char* Input::one(const char* command) { return run_command(lmp_, command); }

void* Atom::extract(const char* name) {
  if (!std::strcmp(name, "type")) return type;
  if (!std::strcmp(name, "x")) return x;
  if (!std::strcmp(name, "id")) return tag;
  return 0;
}

void Error::warning(const char* file, int line, const char* msg) {
  std::fprintf(stderr, "WARNING: %s (%s:%d)\n", msg, file, line);
}

}  // namespace LAMMPS_NS

char* lammps_command(void* handle, char* command) {
  return LAMMPS_NS::run_command(static_cast<LAMMPS_NS::LAMMPS*>(handle), command);
}

void* lammps_extract_global(void* handle, char* name) {
  LAMMPS_NS::LAMMPS* lmp = static_cast<LAMMPS_NS::LAMMPS*>(handle);
  static const char* box[6] = {"boxxlo", "boxylo", "boxzlo", "boxxhi", "boxyhi", "boxzhi"};
  if (!std::strcmp(name, "triclinic")) return &lmp->triclinic;
  for (int k = 0; k < 6; ++k)
    if (!std::strcmp(name, box[k])) return k < 3 ? &lmp->boxlo[k] : &lmp->boxhi[k - 3];
  return 0;
}
