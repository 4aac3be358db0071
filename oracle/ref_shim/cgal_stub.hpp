// Forced-include stand-in for the CGAL types that SAMoS's
// src/system/neighbour_list.cpp names outside its HAS_CGAL guard (the
// triangulation helpers get_opposite / mark_domains, lines 37-112).  They are
// only called from the guarded tessellation code, which this build leaves
// out, so the types need to compile, not to work.  Test infrastructure for
// the reference-source oracle build.
#pragma once
#include <utility>

struct ShimCgalFaceInfo { int nesting_level = -1; };
struct ShimCgalVertex {
  unsigned info() const { return 0; }
};
struct ShimCgalFace {
  ShimCgalVertex* vertex(int) const { return nullptr; }
  ShimCgalFace* neighbor(int) const { return nullptr; }
  ShimCgalFaceInfo& info() { return info_; }
  ShimCgalFaceInfo info_;
};
struct Delaunay {
  typedef ShimCgalFace* Face_handle;
  typedef std::pair<Face_handle, int> Edge;
  typedef ShimCgalFace* All_faces_iterator;
  bool is_constrained(const Edge&) const { return false; }
  All_faces_iterator all_faces_begin() { return nullptr; }
  All_faces_iterator all_faces_end() { return nullptr; }
  Face_handle infinite_face() { return nullptr; }
};
