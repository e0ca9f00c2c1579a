"""Mirror of the reference package ``optix_raycasting`` for the differentiable ray caster."""
