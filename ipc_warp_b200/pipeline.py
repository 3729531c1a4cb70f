"""The per-Newton-iteration contact pipeline as one object.

``ContactPipeline`` is a ready-made host for :class:`ContactBarrierMixin`:
it owns the soup, the force accumulator ``b`` and the step ``h``, and
``iteration(dx)`` runs what RodComplexBC does for contact in one Newton
iteration (dynamic_contacts.py:272-308 with contact.py:539-725):

  1. ``detect_collision()``          BVH refit, EE and PT candidate lists
  2. ``compute_contact_hessian()``   16 triplets per record, force into b,
                                     canonical BSR of the contact Hessian
  3. ``compute_collision_energy()``  barrier energy (double) x h^2
  4. ``collision_free_step(dx)``     CCD step bound for x -= alpha dx
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from . import contact
from .contact import Soup
from .dynamic_contacts import ContactBarrierMixin


@dataclass
class NewtonState:
    """fem/params.py:43-50 (the fields the contact pipeline touches)."""
    x: torch.Tensor
    dx: torch.Tensor


@dataclass
class IterationResult:
    n_ee: int
    n_pt: int
    energy: float
    alpha: float


class ContactPipeline(ContactBarrierMixin):
    def __init__(self, soup: Soup, dhat: float, kappa: float, h: float = 1e-2, exclude_same_body: bool = False):
        contact._thickness = 0.5 * dhat
        contact.buffer = 0.5 * dhat
        self.soup = soup
        self.h = float(h)
        self.contact_stiffness = float(kappa)
        self.states = NewtonState(x=soup.x_transformed, dx=torch.zeros_like(soup.x_transformed))
        self.b = torch.zeros_like(soup.x_transformed)
        ContactBarrierMixin.__init__(self)
        self.disable_self_collision = exclude_same_body
        self.collision_triplets = None
        self.collision_hessian = None

    @staticmethod
    def from_scene(scene, dtype=None, device="cuda", exclude_same_body=False) -> "ContactPipeline":
        soup = Soup.from_numpy(scene.x, scene.edges, scene.triangles, scene.body, xcs=scene.xcs, device=device,
                               dtype=dtype)
        return ContactPipeline(soup, scene.dhat, scene.kappa, exclude_same_body=exclude_same_body)

    def iteration(self, dx: torch.Tensor | None = None) -> IterationResult:
        if dx is not None:
            self.states.dx = dx
        self.detect_collision()
        self.b.zero_()
        self.compute_contact_hessian(detect=False)
        e = self.compute_collision_energy(detect=False)
        alpha = self.line_search_upper_bound()
        return IterationResult(self.n_contacts, self.n_contacts_pt, e, alpha)

    def set_positions(self, x) -> None:
        if isinstance(x, np.ndarray):
            x = torch.from_numpy(x)
        self.soup.x_transformed.copy_(x, non_blocking=True)
