"""Host side of the reference binding, without a GPU: the bound classes are
subclasses of the reference's own core classes, keep their class through
the reference executor's ``_configure`` (which rebinds ``core.__class__``),
and ``register()`` points the reference's registry at them."""
import pytest

from oracle import ref_harness as rh

REF = rh.default_reference_path()
pytestmark = pytest.mark.skipif(REF is None, reason="reference package not importable")


@pytest.mark.parametrize("name", ["implicit_p0_fixed", "explicit"])
def test_bound_class_is_the_reference_class_with_the_b200_step(name):
    rh.import_reference(REF)
    from neuralpom_b200 import reference_binding as rb
    base = rb.reference_core_class(name)
    cls = rb.bound_core_class(name)
    assert issubclass(cls, base) and cls is rb.bound_core_class(name)
    assert cls.run_time_loop is not base.run_time_loop


def test_bound_core_keeps_its_class_through_configure():
    rh.import_reference(REF)
    from neuralpom.hybrid.sparse_physics import SparsePhysics
    from neuralpom_b200 import reference_binding as rb
    core = rh.build_reference_core("implicit_p0_fixed", 12, 10)
    rb.bind(core)
    cls = type(core)
    SparsePhysics("cpu")._configure(core)
    assert type(core) is cls
    assert core.use_triton_elliptic_operator is False      # the executor's other settings still apply
    ex = rb.bind(rh.build_reference_core("explicit", 12, 10))
    SparsePhysics("cpu", core_name="explicit", compiled_kernels=())._configure(ex)
    assert type(ex) is rb.bound_core_class("explicit")
    rb.unbind(core)
    assert type(core) is rb.reference_core_class("implicit_p0_fixed")
    with pytest.raises(TypeError):
        rb.bind(object())


def test_register_points_the_reference_registry_at_the_bound_classes():
    rh.import_reference(REF)
    import neuralpom.core_factory as cf
    from neuralpom_b200 import reference_binding as rb
    saved = dict(cf.CORE_REGISTRY)
    try:
        rb.register()
        for name in ("implicit_p0_fixed", "explicit"):
            assert cf.resolve_core_class(name) is rb.bound_core_class(name)
    finally:
        cf.CORE_REGISTRY.clear()
        cf.CORE_REGISTRY.update(saved)
