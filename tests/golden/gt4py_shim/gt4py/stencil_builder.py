class StencilBuilder:
    pass
