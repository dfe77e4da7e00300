"""Host-side logic of the autograd Functions (no GPU): the upstream image
gradients handed to the binding when some outputs carry no loss."""
import pytest

torch = pytest.importorskip("torch")


def _image_grads():
    try:
        from word2world_b200.renderer import _image_grads as f
    except (ImportError, OSError) as e:  # the extension is not built here
        pytest.skip(f"word2world_b200 not importable: {e}")
    return f


def test_absent_depth_and_alpha_gradients_are_empty():
    f = _image_grads()
    alpha = torch.rand(1, 5, 7)
    g = torch.randn(3, 5, 7)
    c, d, a = f(g, None, None, alpha)
    assert c.data_ptr() == g.data_ptr() and c.is_contiguous()
    assert d.numel() == 0 and a.numel() == 0 and d.dtype == torch.float32


def test_colour_gradient_is_zeros_when_only_depth_has_a_loss():
    f = _image_grads()
    alpha = torch.rand(1, 4, 6)
    gd = torch.randn(1, 6, 4).transpose(1, 2)  # non-contiguous
    c, d, a = f(None, gd, None, alpha)
    assert c.shape == (3, 4, 6) and float(c.abs().sum()) == 0.0
    assert d.is_contiguous() and torch.equal(d, gd)
    assert a.numel() == 0
