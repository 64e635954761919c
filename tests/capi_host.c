/* A plain C caller of the p3d_b200 C ABI: only the entry points that need no
 * device (descriptors, workspace sizes, solver options, error reporting), so
 * that it runs on any host.  Built and run by tests/test_capi.py. */
#include <stdio.h>
#include <string.h>

#include "p3d_b200.h"

int main(void)
{
  p3d_mesh_desc d;
  int rc = p3d_mesh_desc_whole(4, 3, 5, P3D_BC_BIT(P3D_FACE_IMIN, 0), &d);
  printf("desc %d %d %d %d %d %d %d %u %u\n", rc, d.mx, d.gx, d.gy, d.gz, d.ox, d.oz, d.dirichlet, d.global_faces);
  rc = p3d_mesh_desc_whole(0, 3, 5, 0, &d);
  printf("bad_desc %d %s\n", rc, strstr(p3d_last_error(), "bad sizes") ? "msg" : "nomsg");
  int64_t ws = -1;
  rc = p3d_marker_project_workspace(4, 3, 5, P3D_PROJ_Q1, &ws);
  printf("ws_q1 %d %lld\n", rc, (long long)ws);
  rc = p3d_marker_project_workspace(4, 3, 5, P3D_PROJ_P0_HARMONIC, &ws);
  printf("ws_p0 %d %lld\n", rc, (long long)ws);
  p3d_solver_opts o;
  rc = p3d_solver_default_opts(&o);
  int64_t bytes = 0;
  p3d_mesh_desc_whole(32, 32, 32, 0, &d);
  int rc2 = p3d_solver_estimate_bytes(&d, &o, &bytes);
  printf("solver %d %d %d %d\n", rc, o.nlevels, rc2, bytes > 0);
  printf("version %s\n", p3d_version());
  return 0;
}
