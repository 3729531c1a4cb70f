"""ipc_warp_b200: the per-Newton-iteration IPC contact pipeline of ipc_warp
on B200 (sm_100a), behind the reference's Python call surface.

Modules mirror the reference files they replace:
  contact            contact.py            (ContactSolverBase, Contacts, Soup)
  dynamic_contacts   dynamic_contacts.py   (contact_hessian_*, contact_energy_*)
  ccd                ccd/ccd.py, ccd/cubic_roots.py
  bsr                warp.sparse subset    (bsr_from_triplets, bsr_axpy, bsr_mv)
  lbvh               wp.Bvh / wp.Mesh      (LBVH build, refit)
  pipeline           one Newton iteration's contact block
The compute runs in libipcb200.so (include/ipcb.h); there is no CPU path.
"""
__version__ = "0.1.0"
